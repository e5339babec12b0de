/*
 * mms_oracle.c — CPU restatement of the muMatScale CA hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg.  Nothing in the product links, imports or
 * executes it.
 *
 * Pinning: tests/test_oracle_golden.py compares every field this file
 * produces, bit for bit, with dumps of the reference itself (compiled from
 * its own sources under oracle/_ref by oracle/Makefile), and the known
 * answers of the reference's regression tests (tests/testOneGrain.py:25-39).
 *
 * Design: one domain on the reference's halo'd global grid (growth.c:70
 * index on a single subblock).  When NSubblocks is not 1 1 1, each emulated
 * rank r owns the subblock at (r % nx, (r / nx) % ny, r / (nx ny))
 * (MPI_Cart_create dims {nz,ny,nx}, ca_main.c:199-212) and everything that
 * depends on the rank — its rand() stream (ca_main.c:215), its raster-ordered
 * nucleation list, the grain-id offsets (grain.c:892-897) and its interface
 * list with the dc_tmp slot array (growth.c:642-807) — is kept per rank.
 * Halo exchanges need no emulation: every halo read in doiteration is
 * current when it is read (calculate.c:230-343).
 *
 * Floating point: compiled with -ffp-contract=off and evaluated in the same
 * operation order as the reference, so that results are bit-identical to a
 * gcc -O3 x86-64 build of the reference (which emits no FMA).
 */
#define _GNU_SOURCE
#include "mms_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MINF(x, y) (((x) < (y)) ? (x) : (y))
#define MAXF(x, y) (((x) > (y)) ? (x) : (y))

typedef struct {
    double x, y, z;
} dc3;

/* nucleation_t, globals.h:147-160 */
typedef struct {
    double x, y, z;
    size_t cx, cy, cz;
    double gx, gy, gz;
    double threshold;
} nuc_t;

typedef struct {
    struct random_data rd;
    char state[128];
    unsigned seed;
    long ncalls;        /* rand() calls made on this stream */
    long ncalls_presb;  /* calls made before init_sb_nucleation */
    int have_gauss;     /* getRandomGaussian cache, functions.c:380-381 */
    float gauss_next;
    nuc_t *nuc;
    int nnuc, nuc_cap;
    int sbx, sby, sbz;
    /* interface list and dc_tmp (growth.c:642-660), 1-based slots */
    long *list;
    long gindex;
    dc3 *dc_tmp;
    long dc_tmp_size;
    /* nucleation candidates of the current step (grain.c:1297-1318) */
    long *cand;
    long ncand;
} rank_t;

struct mmso {
    mms_params p;
    int gx, gy, gz;
    long sy, sz, N;
    int nranks;
    long sbcells;
    double *ce, *oce, *cl, *fs, *d, *T, *curv;
    dc3 *dc;
    int *gr, *ogr, *lsindex;
    float *thr;
    signed char *mold;
    mms_grain *grains;
    long grains_cap;
    int num_grains;
    uint64_t timestep;
    rank_t *ranks;
    int curv_on;
    long *inj_idx;
    double *inj_rot;
    long ninj;
    int warned;
    int stepped;
    uint64_t *renum;    /* grain renumbering of the last XDMF write */
    int renum_n;
};

/* ---------------------------------------------------------------- RNG ---- */
/* glibc rand() is random() on a TYPE_3 state of 128 bytes; srand(s) is
 * initstate on that state.  random_r keeps one stream per emulated rank. */
static void rng_seed(rank_t *r, unsigned seed)
{
    memset(&r->rd, 0, sizeof r->rd);
    memset(r->state, 0, sizeof r->state);
    initstate_r(seed, r->state, sizeof r->state, &r->rd);
    r->seed = seed;
    r->ncalls = 0;
    r->have_gauss = 0;
    r->gauss_next = 0.0f;
}

static int32_t rng_rand(rank_t *r)
{
    int32_t v;
    random_r(&r->rd, &v);
    r->ncalls++;
    return v;
}

/* getRandScale, functions.c:440-445 */
static float rng_scale(rank_t *r) { return (float)rng_rand(r) / (float)RAND_MAX; }

/* getRandomGaussian, functions.c:376-406 (Marsaglia polar, one cached value) */
static float rng_gauss(rank_t *r)
{
    if (r->have_gauss) {
        r->have_gauss = 0;
        return r->gauss_next;
    }
    float n0, n1, s;
    do {
        n0 = ((float)rng_rand(r) / (float)(RAND_MAX / 2.0)) - 1.0;
        n1 = ((float)rng_rand(r) / (float)(RAND_MAX / 2.0)) - 1.0;
        s = n0 * n0 + n1 * n1;
    } while (s >= 1.0 || s == 0);
    float multiplier = sqrtf(-2.0 * log(s) / s);
    float val = n0 * multiplier;
    r->gauss_next = n1 * multiplier;
    r->have_gauss = 1;
    return val;
}

void mmso_rand_sequence(unsigned seed, int n, int32_t *out)
{
    rank_t r;
    rng_seed(&r, seed);
    for (int i = 0; i < n; i++) out[i] = rng_rand(&r);
}

/* --------------------------------------------------------- geometry ------ */
static long cidx(const mmso *o, long i, long j, long k) { return k * o->sz + j * o->sy + i; }

/* realcoord2scoord, functions.c:91-107 */
static void real2cell(const mmso *o, double x, double y, double z, size_t *i, size_t *j, size_t *k)
{
    const mms_params *p = &o->p;
    x = x - p->origin_offset[0] + p->cellSize * 0.1;
    y = y - p->origin_offset[1] + p->cellSize * 0.1;
    z = z - p->origin_offset[2] + p->cellSize * 0.1;
    *i = (size_t)(x / p->cellSize);
    *j = (size_t)(y / p->cellSize);
    *k = (size_t)(z / p->cellSize);
}

/* CELLCOORD2REALCOORDn, functions.h:284-286 */
static double cell2real(const mmso *o, int axis, double i)
{
    return o->p.origin_offset[axis] + (i + 0.5) * o->p.cellSize;
}

/* sbID_from_sbcoords / sbID_from_realcoords, functions.c:271-352 (pad case) */
static int rank_of_cell(const mmso *o, size_t cx, size_t cy, size_t cz)
{
    const mms_params *p = &o->p;
    long x = (long)(cx / (size_t)p->gsdimx), y = (long)(cy / (size_t)p->gsdimy),
         z = (long)(cz / (size_t)p->gsdimz);
    if (!p->padBndyX) x = (x + p->gnsbx) % p->gnsbx;
    if (!p->padBndyY) y = (y + p->gnsby) % p->gnsby;
    if (!p->padBndyZ) z = (z + p->gnsbz) % p->gnsbz;
    if (x < 0 || y < 0 || z < 0 || x >= p->gnsbx || y >= p->gnsby || z >= p->gnsbz) return -1;
    return (int)(x + y * p->gnsbx + z * p->gnsbx * p->gnsby);
}

/* global halo'd cell of rank-local halo'd coordinates */
static long rank_cell(const mmso *o, const rank_t *r, long i, long j, long k)
{
    return cidx(o, r->sbx * (long)o->p.gsdimx + i, r->sby * (long)o->p.gsdimy + j,
                r->sbz * (long)o->p.gsdimz + k);
}

/* ------------------------------------------------------ temperature ----- */
/* direct_temp_calc, temperature.c:23-126, at global halo'd cell (I,J,K) */
static double temp_at(const mmso *o, long I, long J, long K, uint64_t ts)
{
    const mms_params *p = &o->p;
    double sim_time = ts * p->ts_delt;
    double T = 0.0;
    if (p->thermal_ana == 0 && p->gradient == 0) {
        T = p->initialTemperature - sim_time * p->cool_rate;
    } else {
        double rx = cell2real(o, 0, (double)(int)I), ry = cell2real(o, 1, (double)(int)J),
               rz = cell2real(o, 2, (double)(int)K);
        if (!p->am) {
            double axis = ((o->gz == 1) ? ry : rz) - p->cellSize * 0.5;
            double tgrad = p->gradient + p->grad_coef * sim_time;
            double v = p->velocity + p->velo_coef * sim_time;
            double vt = 0.5 * (v + p->velocity) * sim_time;
            T = p->initialTemperature + tgrad * (axis - vt);
        } else if (p->thermal_ana == 1) {
            double lv = p->lv;
            double invlv = 1. / lv;
            double ls = p->lsd / (2. * 1.414);
            double xlen = p->gnsbx * p->gsdimx * p->cellSize;
            xlen = xlen + p->lsd;
            double tline = xlen * invlv;
            double tpause = 1.5e-4 * invlv;
            tline = tline + tpause;
            double trackno = 0;
            if (p->amtracks > 1) trackno = floor(sim_time / tline);
            double xnow = p->x0 + (sim_time - trackno * tline) * lv;
            double ynow = p->y0 + trackno * p->lhs;
            double znow = p->z0;
            double lpow = p->lpow;
            double lx = rx - xnow, ly = ry - ynow, lz = rz - znow;
            if (rz <= znow + p->cellSize) {
                int nt = 400;
                double lt, Tlocal, Tfront, Tinteg = 0.0;
                double pi15 = 5.568328;
                double lalpha = p->lthcon / (p->rho * p->lcp);
                double tsteady = 20 * lalpha * invlv * invlv;
                double ldt = tsteady / nt;
                if (sim_time < 1e-4) lpow = 0;
                for (int i = 0; i < nt; i++) {
                    lt = (0.5 + i) * ldt;
                    Tlocal = sqrt(lalpha * lt) * (ls * ls + 4. * lalpha * lt);
                    Tinteg += ldt *
                              exp(-((lx + lv * lt) * (lx + lv * lt) + ly * ly) /
                                      (ls * ls + 4. * lalpha * lt) -
                                  (lz * lz / (4. * lalpha * lt))) /
                              Tlocal;
                }
                Tfront = p->lab * lpow * lalpha / (pi15 * p->lthcon);
                T = p->liniT + Tfront * Tinteg;
            } else {
                T = 0.0;
            }
        }
    }
    return T;
}

/* tempUpdateSB_int, temperature.c:218-272 */
static void temp_update(mmso *o)
{
    for (long K = 0; K < o->gz + 2; K++)
        for (long J = 0; J < o->gy + 2; J++)
            for (long I = 0; I < o->gx + 2; I++) {
                long c = cidx(o, I, J, K);
                o->T[c] = temp_at(o, I, J, K, o->timestep);
                if (o->p.thermal_ana && o->T[c] > o->p.liquidusTemp) o->lsindex[c] = 1;
            }
}

/* ---------------------------------------------------------- grains ------ */
/* setNucOrientation, grain.c:117-130 */
static void set_orientation(const mmso *o, rank_t *r, nuc_t *nuc)
{
    nuc->gx = nuc->gy = nuc->gz = 0.0;
    if (o->p.gnUseOrientation) {
        float acon = 4.0;
        nuc->gx = M_PI / acon - 2 * (M_PI / acon * rng_scale(r));
        nuc->gy = M_PI / acon - 2 * (M_PI / acon * rng_scale(r));
        nuc->gz = M_PI / acon - 2 * (M_PI / acon * rng_scale(r));
    }
}

/* nucleate_grain, grain.c:300-344 */
static void make_grain(const mmso *o, const nuc_t *nuc, mms_grain *g)
{
    double a0 = nuc->gx, a1 = nuc->gy, a2 = nuc->gz;
    double c0 = cos(a0), s0 = sin(a0), c1 = cos(a1), s1 = sin(a1), c2 = cos(a2), s2 = sin(a2);
    g->rotang[0] = nuc->gx;
    g->rotang[1] = nuc->gy;
    g->rotang[2] = nuc->gz;
    g->rotmat[0][0] = c2 * c0 - s2 * s1 * s0;
    g->rotmat[1][0] = c2 * s0 + s2 * c1 * c0;
    g->rotmat[2][0] = s2 * s1;
    g->rotmat[0][1] = -1. * s2 * c0 - c2 * c1 * s0;
    g->rotmat[1][1] = -1. * s2 * s0 + c2 * c1 * c0;
    g->rotmat[2][1] = c2 * s1;
    g->rotmat[0][2] = s1 * s0;
    g->rotmat[1][2] = -1. * s1 * c0;
    g->rotmat[2][2] = c1;
    g->nuc_x = nuc->x;
    g->nuc_y = nuc->y;
    g->nuc_z = nuc->z;
    g->nuc_timestep = o->timestep;
    g->nuc_threshold = nuc->threshold;
}

static void rank_add_nuc(rank_t *r, const nuc_t *n)
{
    if (r->nnuc + 1 > r->nuc_cap) {
        r->nuc_cap = r->nuc_cap ? 2 * r->nuc_cap : 16;
        r->nuc = (nuc_t *)realloc(r->nuc, sizeof(nuc_t) * (size_t)r->nuc_cap);
    }
    r->nuc[r->nnuc++] = *n;
}

/* ------------------------------------------------------------ setup ----- */
typedef void (*select_fn)(mmso *o, rank_t *r, size_t index, void *ud);

/* distribute_nucleations (Knuth Algorithm S), grain.c:250-296 */
static void distribute(mmso *o, rank_t *r, size_t nc, size_t num, select_fn fn, void *ud)
{
    size_t n = MINF(num, nc);
    size_t N = nc;
    size_t t = 0, m = 0, idx = 0;
    if (n == 0) return;
    do {
        double U = rng_scale(r);
        if ((N - t) * U >= (n - m)) {
            t++;
        } else {
            fn(o, r, idx, ud);
            t++;
            m++;
        }
        idx++;
    } while (m < n);
}

typedef struct {
    size_t minCell[3], maxCell[3];
    double threshold;
    nuc_t *out;
    size_t nout;
} vol_ud;

/* select_nuc_volume, grain.c:173-210 */
static void select_volume(mmso *o, rank_t *r, size_t index, void *vud)
{
    vol_ud *v = (vol_ud *)vud;
    size_t nx = v->maxCell[0] - v->minCell[0];
    size_t ny = v->maxCell[1] - v->minCell[1];
    nuc_t nuc;
    nuc.cx = v->minCell[0] + index % nx;
    nuc.cy = v->minCell[1] + (index % (nx * ny)) / nx;
    nuc.cz = v->minCell[2] + index / (nx * ny);
    nuc.threshold = v->threshold;
    set_orientation(o, r, &nuc);
    nuc.x = cell2real(o, 0, (double)nuc.cx);
    nuc.y = cell2real(o, 1, (double)nuc.cy);
    nuc.z = cell2real(o, 2, (double)nuc.cz);
    v->out[v->nout++] = nuc;
}

typedef struct {
    long *cells;
    double center, sigma;
} thr_ud;

/* genRandomThreshold, grain.c:140-154 */
static float random_threshold(rank_t *r, double center, double sigma)
{
    float t = 0.0;
    do {
        t = (float)(sigma * rng_gauss(r) + center);
    } while ((t < 1.0e-5) || (fabs(t - center) > (6.0 * sigma)));
    return t;
}

/* select_if_not_fixed, grain.c:225-237 */
static void select_threshold(mmso *o, rank_t *r, size_t index, void *vud)
{
    thr_ud *u = (thr_ud *)vud;
    long c = u->cells[index];
    if (o->thr[c] == INFINITY) o->thr[c] = random_threshold(r, u->center, u->sigma);
}

/* init_nucleation_sites, grain.c:602-713 (rank 0) */
static void init_nucleation_sites(mmso *o)
{
    const mms_params *p = &o->p;
    rank_t *r0 = &o->ranks[0];
    size_t total = (size_t)p->n_fixed_nucs;
    nuc_t *all = (nuc_t *)malloc(sizeof(nuc_t) * (total ? total : 1));
    size_t nall = 0;
    for (int f = 0; f < p->n_fixed_nucs; f++) {
        const mms_fixed_nuc *fn = &p->fixed_nucs[f];
        nuc_t n;
        memset(&n, 0, sizeof n);
        n.x = fn->x;
        n.y = fn->y;
        n.z = fn->z;
        n.gx = (M_PI / 180.0) * fn->ax;
        n.gy = (M_PI / 180.0) * fn->ay;
        n.gz = (M_PI / 180.0) * fn->az;
        n.threshold = fn->threshold;
        real2cell(o, n.x, n.y, n.z, &n.cx, &n.cy, &n.cz);
        all[nall++] = n;
    }
    for (int v = 0; v < p->n_nuc_volumes; v++) {
        mms_nuc_volume nv = p->nuc_volumes[v];
        nv.minx = MAXF(nv.minx, p->origin_offset[0]);
        nv.maxx = MINF(nv.maxx, p->origin_offset[0] + (o->gx * p->cellSize));
        nv.miny = MAXF(nv.miny, p->origin_offset[1]);
        nv.maxy = MINF(nv.maxy, p->origin_offset[1] + (o->gy * p->cellSize));
        nv.minz = MAXF(nv.minz, p->origin_offset[2]);
        nv.maxz = MINF(nv.maxz, p->origin_offset[2] + (o->gz * p->cellSize));
        vol_ud ud;
        memset(&ud, 0, sizeof ud);
        real2cell(o, nv.minx, nv.miny, nv.minz, &ud.minCell[0], &ud.minCell[1], &ud.minCell[2]);
        real2cell(o, nv.maxx, nv.maxy, nv.maxz, &ud.maxCell[0], &ud.maxCell[1], &ud.maxCell[2]);
        size_t count = (ud.maxCell[0] - ud.minCell[0]) * (ud.maxCell[1] - ud.minCell[1]) *
                       (ud.maxCell[2] - ud.minCell[2]);
        size_t max_nucs = count * nv.density;
        all = (nuc_t *)realloc(all, sizeof(nuc_t) * (nall + max_nucs + 1));
        ud.threshold = nv.threshold;
        ud.out = all + nall;
        distribute(o, r0, count, max_nucs, select_volume, &ud);
        nall += ud.nout;
    }
    for (size_t i = 0; i < nall; i++) {
        size_t cx, cy, cz;
        real2cell(o, all[i].x, all[i].y, all[i].z, &cx, &cy, &cz);
        int sb = rank_of_cell(o, cx, cy, cz);
        if (sb >= 0) rank_add_nuc(&o->ranks[sb], &all[i]);
    }
    free(all);
}

/* init_sb_nucleation, grain.c:930-1010, for one emulated rank */
static void init_sb_nucleation(mmso *o, rank_t *r)
{
    const mms_params *p = &o->p;
    for (int n = 0; n < r->nnuc; n++) {
        const nuc_t *nu = &r->nuc[n];
        long x = 1 + (long)(nu->cx % (size_t)p->gsdimx);
        long y = 1 + (long)(nu->cy % (size_t)p->gsdimy);
        long z = 1 + (long)(nu->cz % (size_t)p->gsdimz);
        long c = rank_cell(o, r, x, y, z);
        if (!o->mold[c]) o->thr[c] = nu->threshold;
    }
    long *suf = (long *)malloc(sizeof(long) * (size_t)o->sbcells);
    long *vol = (long *)malloc(sizeof(long) * (size_t)o->sbcells);
    size_t s = 0, v = 0;
    for (long z = 1; z <= p->gsdimz; z++)
        for (long y = 1; y <= p->gsdimy; y++)
            for (long x = 1; x <= p->gsdimx; x++) {
                long c = rank_cell(o, r, x, y, z);
                if (!o->mold[c]) {
                    vol[v++] = c;
                    int surf = o->mold[c - 1] + o->mold[c + 1] + o->mold[c - o->sy] +
                               o->mold[c + o->sy] + o->mold[c - o->sz] + o->mold[c + o->sz];
                    if (surf) suf[s++] = c;
                }
            }
    thr_ud ud = {vol, p->gnGaussCenter, p->gnGaussSigma};
    size_t count = p->maxGrainDensity * (v * pow(p->cellSize, 3.0));
    distribute(o, r, v, count, select_threshold, &ud);
    if (p->doSurfaceNuc && (p->maxGrainDensitySurf > 0.0)) {
        ud.cells = suf;
        ud.center = p->gnGaussCenterSurf;
        ud.sigma = p->gnGaussSigmaSurf;
        count = p->maxGrainDensitySurf * (s * pow(p->cellSize, 2.0));
        distribute(o, r, s, count, select_threshold, &ud);
    }
    free(suf);
    free(vol);
}

/* ------------------------------------------------------ create/destroy -- */
mmso *mmso_create(const mms_params *pin, int *status)
{
    mms_params p = *pin;
    *status = MMS_OK;
    if (p.gnsbx < 1 || p.gnsby < 1 || p.gnsbz < 1 || p.gsdimx < 1 || p.gsdimy < 1 ||
        p.gsdimz < 1 || p.cellSize <= 0 || p.ts_delt <= 0) {
        *status = MMS_ERR_ARG;
        return NULL;
    }
    if ((!p.padBndyX && p.gnsbx > 1) || (!p.padBndyY && p.gnsby > 1) ||
        (!p.padBndyZ && p.gnsbz > 1)) {
        *status = MMS_ERR_ARG; /* periodic exchange between subblocks: not supported */
        return NULL;
    }
    if (p.am && p.thermal_ana != 1) {
        *status = MMS_ERR_ARG;
        return NULL;
    }
    /* Courant check, growth.c:38-50 */
    double dtx = p.ts_delt / (p.cellSize * p.cellSize);
    if (p.Dsol * dtx > p.courant_limit || p.Dliq * dtx > p.courant_limit) {
        *status = MMS_ERR_COURANT;
        return NULL;
    }
    mmso *o = (mmso *)calloc(1, sizeof(mmso));
    o->p = p;
    o->p.fixed_nucs = NULL;
    o->p.nuc_volumes = NULL;
    o->gx = p.gnsbx * p.gsdimx;
    o->gy = p.gnsby * p.gsdimy;
    o->gz = p.gnsbz * p.gsdimz;
    o->sy = o->gx + 2;
    o->sz = (long)(o->gx + 2) * (o->gy + 2);
    o->N = o->sz * (o->gz + 2);
    o->nranks = p.gnsbx * p.gnsby * p.gnsbz;
    o->sbcells = (long)p.gsdimx * p.gsdimy * p.gsdimz;
    long N = o->N;
    o->ce = (double *)calloc(N, sizeof(double));
    o->oce = (double *)calloc(N, sizeof(double));
    o->cl = (double *)calloc(N, sizeof(double));
    o->fs = (double *)calloc(N, sizeof(double));
    o->d = (double *)calloc(N, sizeof(double));
    o->T = (double *)calloc(N, sizeof(double));
    o->curv = (double *)calloc(N, sizeof(double));
    o->dc = (dc3 *)calloc(N, sizeof(dc3));
    o->gr = (int *)calloc(N, sizeof(int));
    o->ogr = (int *)calloc(N, sizeof(int));
    o->lsindex = (int *)calloc(N, sizeof(int));
    o->thr = (float *)calloc(N, sizeof(float));
    o->mold = (signed char *)calloc(N, 1);
    o->grains_cap = 1024;
    o->grains = (mms_grain *)calloc((size_t)o->grains_cap, sizeof(mms_grain));
    o->num_grains = 1; /* the "zero" grain, read_ctrl.c:51 */
    o->ranks = (rank_t *)calloc((size_t)o->nranks, sizeof(rank_t));
    for (int r = 0; r < o->nranks; r++) {
        rank_t *rk = &o->ranks[r];
        rk->sbx = r % p.gnsbx;
        rk->sby = (r / p.gnsbx) % p.gnsby;
        rk->sbz = r / (p.gnsbx * p.gnsby);
        rng_seed(rk, (unsigned)r + 1 + p.base_random_seed);
        rk->list = (long *)calloc((size_t)o->sbcells + 2, sizeof(long));
        rk->cand = (long *)calloc((size_t)o->sbcells + 1, sizeof(long));
    }
    /* SetupInitialConditions, setup.c:41-94 */
    for (long c = 0; c < N; c++) {
        o->thr[c] = INFINITY;
        o->ce[c] = o->cl[c] = p.Cinit;
    }
    /* tempPrepareSB_int, temperature.c:155-215 */
    for (long K = 0; K < o->gz + 2; K++)
        for (long J = 0; J < o->gy + 2; J++)
            for (long I = 0; I < o->gx + 2; I++) {
                long c = cidx(o, I, J, K);
                o->T[c] = temp_at(o, I, J, K, 0);
                if (p.am) o->lsindex[c] = (o->T[c] >= p.liquidusTemp) ? 1 : 0;
                int m = 0;
                if (p.padBndyX && (I == 0 || I == o->gx + 1)) m = 1;
                if (p.padBndyY && (J == 0 || J == o->gy + 1)) m = 1;
                if (p.padBndyZ && (K == 0 || K == o->gz + 1)) m = 1;
                o->mold[c] = (signed char)m;
            }
    o->p.fixed_nucs = pin->fixed_nucs;
    o->p.nuc_volumes = pin->nuc_volumes;
    init_nucleation_sites(o);
    o->p.fixed_nucs = NULL;
    o->p.nuc_volumes = NULL;
    for (int r = 0; r < o->nranks; r++) {
        o->ranks[r].ncalls_presb = o->ranks[r].ncalls;
        init_sb_nucleation(o, &o->ranks[r]);
    }
    return o;
}

void mmso_destroy(mmso *o)
{
    if (!o) return;
    free(o->ce); free(o->oce); free(o->cl); free(o->fs); free(o->d); free(o->T);
    free(o->curv); free(o->dc); free(o->gr); free(o->ogr); free(o->lsindex);
    free(o->thr); free(o->mold); free(o->grains); free(o->inj_idx); free(o->inj_rot); free(o->renum);
    for (int r = 0; r < o->nranks; r++) {
        free(o->ranks[r].nuc);
        free(o->ranks[r].list);
        free(o->ranks[r].dc_tmp);
        free(o->ranks[r].cand);
    }
    free(o->ranks);
    free(o);
}

/* Site injection: replaces init_sb_nucleation's draws (as the reference's
 * --wrap=init_sb_nucleation hook does): thresholds reset to +inf, listed
 * interior cells get their threshold, and each rank's stream is rewound to
 * where init_sb_nucleation would have started drawing. */
int mmso_set_sites(mmso *o, int64_t n, const int32_t *gxyz, const float *thr)
{
    if (o->stepped) return MMS_ERR_STATE;
    for (long c = 0; c < o->N; c++) o->thr[c] = INFINITY;
    for (int64_t s = 0; s < n; s++) {
        long x = gxyz[3 * s], y = gxyz[3 * s + 1], z = gxyz[3 * s + 2];
        if (x < 0 || y < 0 || z < 0 || x >= o->gx || y >= o->gy || z >= o->gz) return MMS_ERR_ARG;
        long c = cidx(o, x + 1, y + 1, z + 1);
        if (!o->mold[c]) o->thr[c] = thr[s];
    }
    for (int r = 0; r < o->nranks; r++) {
        rank_t *rk = &o->ranks[r];
        long keep = rk->ncalls_presb;
        rng_seed(rk, rk->seed);
        while (rk->ncalls < keep) rng_rand(rk);
    }
    return MMS_OK;
}

static int cmp_long(const void *a, const void *b)
{
    long x = *(const long *)a, y = *(const long *)b;
    return (x > y) - (x < y);
}

/* Pre-filled microstructure (the library's mms_set_grains): grains 1..n
 * with the given rotation matrices; nucleated grains continue from n+1. */
int mmso_set_grains(mmso *o, int n, const double *rot9)
{
    if (n < 0 || o->stepped || (uint64_t)n + 1 > o->p.maxTotalGrains + 1) return MMS_ERR_ARG;
    if (n + 1 > o->grains_cap) {
        long nc = n + 1024;
        o->grains = (mms_grain *)realloc(o->grains, sizeof(mms_grain) * (size_t)nc);
        o->grains_cap = nc;
    }
    memset(o->grains + 1, 0, sizeof(mms_grain) * (size_t)(o->grains_cap - 1));
    for (int g = 0; g < n; g++)
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) o->grains[g + 1].rotmat[a][b] = rot9[9 * g + 3 * a + b];
    o->num_grains = n + 1;
    return MMS_OK;
}

/* Field upload in the halo'd layout (ce, cl, fs, gr, dc). */
int mmso_set_field(mmso *o, int field, const void *in)
{
    size_t N = (size_t)o->N;
    switch (field) {
    case MMS_FIELD_CE: memcpy(o->ce, in, N * sizeof(double)); break;
    case MMS_FIELD_CL: memcpy(o->cl, in, N * sizeof(double)); break;
    case MMS_FIELD_FS: memcpy(o->fs, in, N * sizeof(double)); break;
    case MMS_FIELD_GR: memcpy(o->gr, in, N * sizeof(int)); break;
    case MMS_FIELD_DC: memcpy(o->dc, in, N * sizeof(dc3)); break;
    default: return MMS_ERR_ARG;
    }
    return MMS_OK;
}

int mmso_set_site_orientations(mmso *o, int64_t n, const int32_t *gxyz, const double *rot9)
{
    free(o->inj_idx);
    free(o->inj_rot);
    o->ninj = n;
    o->inj_idx = (long *)malloc(sizeof(long) * 2 * (size_t)(n ? n : 1));
    o->inj_rot = (double *)malloc(sizeof(double) * 9 * (size_t)(n ? n : 1));
    /* sort (cell, original index) pairs so lookups are binary searches; the
     * first listed entry of a cell wins, like the hook's linear search */
    for (int64_t s = 0; s < n; s++) {
        long x = gxyz[3 * s], y = gxyz[3 * s + 1], z = gxyz[3 * s + 2];
        o->inj_idx[2 * s] = (z * o->gy + y) * (long)o->gx + x;
        o->inj_idx[2 * s + 1] = s;
    }
    qsort(o->inj_idx, (size_t)n, 2 * sizeof(long), cmp_long);
    double *tmp = (double *)malloc(sizeof(double) * 9 * (size_t)(n ? n : 1));
    for (int64_t s = 0; s < n; s++) {
        /* stable: among equal keys keep the smallest original index first */
        memcpy(tmp + 9 * s, rot9 + 9 * o->inj_idx[2 * s + 1], 9 * sizeof(double));
    }
    for (int64_t s = 1; s < n; s++) {
        if (o->inj_idx[2 * s] == o->inj_idx[2 * (s - 1)] &&
            o->inj_idx[2 * s + 1] < o->inj_idx[2 * (s - 1) + 1]) {
            /* qsort is not stable; fix order of duplicates */
            long t0 = o->inj_idx[2 * s + 1];
            o->inj_idx[2 * s + 1] = o->inj_idx[2 * (s - 1) + 1];
            o->inj_idx[2 * (s - 1) + 1] = t0;
            memcpy(tmp + 9 * s, rot9 + 9 * o->inj_idx[2 * s + 1], 9 * sizeof(double));
            memcpy(tmp + 9 * (s - 1), rot9 + 9 * o->inj_idx[2 * (s - 1) + 1], 9 * sizeof(double));
        }
    }
    memcpy(o->inj_rot, tmp, sizeof(double) * 9 * (size_t)(n ? n : 1));
    free(tmp);
    return MMS_OK;
}

void mmso_enable_curvature(mmso *o, int on) { o->curv_on = on; }

/* --------------------------------------------------------------- step --- */
/* cell_nucleation, grain.c:1043-1326 (NUC_SEP, !NUC_THREELIST branch
 * 1222-1318).  addNewGrain's per-rank cap (grain.c:100-107) only limits
 * which locations are stored: the count handed to activateNewGrains is the
 * uncapped nindex2 (grain.c:1318), so a binding cap always ends in
 * createGrains' error (grain.c:363-366); see activation(). */
static void nucleation(mmso *o)
{
    const mms_params *p = &o->p;
    double sim_time = o->timestep * p->ts_delt;
    for (int r = 0; r < o->nranks; r++) {
        rank_t *rk = &o->ranks[r];
        rk->ncand = 0;
        for (long k = 1; k <= p->gsdimz; k++)
            for (long j = 1; j <= p->gsdimy; j++)
                for (long i = 1; i <= p->gsdimx; i++) {
                    long c = rank_cell(o, rk, i, j, k);
                    double Ttemp = o->T[c];
                    int layerno = 1, initnuc = 1;
                    if (p->am) {
                        if (p->amlayer == 1) layerno = 1;
                        else if (p->amlayer > 1 && o->lsindex[c] == 1) layerno = 1;
                        else layerno = 0;
                        if (sim_time <= 1e-4) initnuc = 1;
                        else if (Ttemp >= p->solidusTemp) initnuc = 1;
                        else initnuc = 0;
                    }
                    if (o->gr[c] <= 0 && layerno && initnuc) {
                        double Tunder = p->liquidusTemp - Ttemp;
                        double m = p->m_solute0_a * Ttemp * Ttemp + p->m_solute0_b * Ttemp +
                                   p->m_solute0_c;
                        Tunder += m * (o->cl[c] - p->Cinit);
                        if (Tunder > o->thr[c]) rk->cand[rk->ncand++] = c;
                    }
                }
    }
}

static const double *injected_rot(const mmso *o, long gcell)
{
    long lo = 0, hi = o->ninj - 1;
    while (lo <= hi) {
        long mid = (lo + hi) / 2;
        long key = o->inj_idx[2 * mid];
        if (key == gcell) {
            while (mid > 0 && o->inj_idx[2 * (mid - 1)] == gcell) mid--;
            return o->inj_rot + 9 * mid;
        }
        if (key < gcell) lo = mid + 1;
        else hi = mid - 1;
    }
    return NULL;
}

/* activateNewGrains + createGrains, grain.c:347-425 and 840-916.  When the
 * candidates exceed the room left under MaxTotGrains the reference caps
 * new_activations but still creates every candidate's grain, and
 * createGrains stops with an error at the first id above MaxTotGrains
 * (grain.c:363-366); that is reported here as MMS_ERR_GRAIN_OVERFLOW. */
static int activation(mmso *o)
{
    const mms_params *p = &o->p;
    int nr = o->nranks;
    long *counts = (long *)calloc((size_t)nr, sizeof(long));
    long new_act = 0;
    for (int r = 0; r < nr; r++) {
        counts[r] = o->ranks[r].ncand;
        new_act += counts[r];
    }
    if ((uint64_t)(o->num_grains + new_act) > (p->maxTotalGrains + 1)) {
        free(counts);
        return MMS_ERR_GRAIN_OVERFLOW;
    }
    int status = MMS_OK;
    if (new_act) {
        int before = o->num_grains;
        long base = o->num_grains;
        long top = base;
        for (int r = 0; r < nr; r++) top += counts[r];
        if (top > o->grains_cap) {
            long nc = o->grains_cap;
            while (nc < top) nc *= 2;
            o->grains = (mms_grain *)realloc(o->grains, sizeof(mms_grain) * (size_t)nc);
            memset(o->grains + o->grains_cap, 0, sizeof(mms_grain) * (size_t)(nc - o->grains_cap));
            o->grains_cap = nc;
        }
        for (int r = 0; r < nr; r++) {
            rank_t *rk = &o->ranks[r];
            for (long g = 0; g < counts[r]; g++) {
                long gr_num = base + g;
                if ((uint64_t)gr_num > p->maxTotalGrains) {
                    status = MMS_ERR_GRAIN_OVERFLOW;
                    break;
                }
                long c = rk->cand[g];
                long K = c / o->sz, J = (c % o->sz) / o->sy, I = c % o->sy;
                size_t x = (size_t)(I - 1), y = (size_t)(J - 1), z = (size_t)(K - 1);
                o->gr[c] = (int)gr_num;
                nuc_t nuc;
                int found = 0;
                for (int j = 0; j < rk->nnuc; j++) {
                    if (rk->nuc[j].cx == x && rk->nuc[j].cy == y && rk->nuc[j].cz == z) {
                        nuc = rk->nuc[j];
                        found = 1;
                        break;
                    }
                }
                if (!found) {
                    nuc.cx = x;
                    nuc.cy = y;
                    nuc.cz = z;
                    nuc.threshold = o->thr[c];
                    nuc.x = cell2real(o, 0, (double)x);
                    nuc.y = cell2real(o, 1, (double)y);
                    nuc.z = cell2real(o, 2, (double)z);
                    set_orientation(o, rk, &nuc);
                }
                make_grain(o, &nuc, &o->grains[gr_num]);
            }
            base += counts[r];
            if (status) break;
        }
        /* orientation injection, applied after the Allgatherv like the hook */
        if (o->ninj > 0) {
            for (long id = before; id < base && id < o->grains_cap; id++) {
                mms_grain *g = &o->grains[id];
                size_t cx, cy, cz;
                real2cell(o, g->nuc_x, g->nuc_y, g->nuc_z, &cx, &cy, &cz);
                long key = ((long)cz * o->gy + (long)cy) * (long)o->gx + (long)cx;
                const double *rot = injected_rot(o, key);
                if (rot) memcpy(&g->rotmat[0][0], rot, 9 * sizeof(double));
            }
        }
    }
    o->num_grains += (int)new_act;
    free(counts);
    return status;
}

/* sb_diffuse_alloy_decentered, growth.c:29-170 */
static int diffuse(mmso *o)
{
    const mms_params *p = &o->p;
    double dtx = p->ts_delt / (p->cellSize * p->cellSize);
    double rs = (p->Dsol * dtx);
    double rl = (p->Dliq * dtx);
    const double *fs = o->fs, *cl = o->cl;
    const signed char *mold = o->mold;
    double *ce = o->ce;
    int status = MMS_OK;
    for (long k = 1; k <= o->gz; k++)
        for (long j = 1; j <= o->gy; j++)
            for (long i = 1; i <= o->gx; i++) {
                long idx = cidx(o, i, j, k);
                double nbsum = 0;
                double conc = cl[idx];
                double lspfs = fs[idx];
                const long nb[6] = {idx + 1, idx - 1, idx + o->sy, idx - o->sy, idx + o->sz, idx - o->sz};
                for (int n = 0; n < 6; n++) {
                    double fs_av = 0.5 * (lspfs + fs[nb[n]]);
                    double r = (rs * fs_av + rl * (1 - fs_av)) * (1 - mold[nb[n]]);
                    double cn = cl[nb[n]];
                    nbsum += r * (cn - conc);
                }
                ce[idx] += nbsum;
                if (ce[idx] < 0) status = MMS_ERR_NEGATIVE_CE;
            }
    return status;
}

/* sb_curvature, curvature.c:30-405, over each rank's local range */
static void curvature(mmso *o)
{
    const mms_params *p = &o->p;
    const double *fs = o->fs;
    const int alpha = 2, beta = 4;
    const long jgap = o->sy, kgap = o->sz;
    for (int r = 0; r < o->nranks; r++) {
        rank_t *rk = &o->ranks[r];
        int dimx = p->gsdimx, dimy = p->gsdimy, dimz = p->gsdimz;
        for (int k = 2; k <= dimz - 1; k++)
            for (int j = 2; j <= dimy - 1; j++)
                for (int i = 2; i <= dimx - 1; i++) {
                    long idx = rank_cell(o, rk, i, j, k);
                    o->curv[idx] = 0.0;
                    if (o->mold[idx] || o->gr[idx] <= 0 || fs[idx] == 0) continue;
                    int nbindex = o->gr[idx + 1] + o->gr[idx + jgap] + o->gr[idx - 1] +
                                  o->gr[idx - jgap] + o->gr[idx + kgap] + o->gr[idx - kgap];
                    if (!nbindex) continue;
                    long idl = idx + 1, idr = idx - 1, idf = idx + jgap, idb = idx - jgap;
                    long idu = idx + kgap, idd = idx - kgap;
                    long idur = idr + kgap, idul = idl + kgap, iddr = idr - kgap, iddl = idl - kgap;
                    long idfr = idf - 1, idfl = idf + 1, idbr = idb - 1, idbl = idb + 1;
                    long idub = idb + kgap, iduf = idf + kgap, iddf = idf - kgap, iddb = idb - kgap;
                    long idufr = iduf - 1, idufl = iduf + 1, idubr = idub - 1, idubl = idub + 1;
                    long iddbr = iddb - 1, iddbl = iddb + 1, iddfr = iddf - 1, iddfl = iddf + 1;
                    double fsl = (fs[idufl] + fs[idubl] + fs[iddbl] + fs[iddfl] +
                                  alpha * (fs[idul] + fs[iddl] + fs[idfl] + fs[idbl]) +
                                  beta * fs[idl]) / (1 + 4 * alpha + beta);
                    double fsr = (fs[idufr] + fs[idubr] + fs[iddbr] + fs[iddfr] +
                                  alpha * (fs[idur] + fs[iddr] + fs[idfr] + fs[idbr]) +
                                  beta * fs[idr]) / (1 + 4 * alpha + beta);
                    double fsf = (fs[idufl] + fs[idufr] + fs[iddfr] + fs[iddfl] +
                                  alpha * (fs[idfl] + fs[idfr] + fs[iduf] + fs[iddf]) +
                                  beta * fs[idf]) / (1 + 4 * alpha + beta);
                    double fsb = (fs[idubr] + fs[idubl] + fs[iddbl] + fs[iddbr] +
                                  alpha * (fs[idbl] + fs[idbr] + fs[idub] + fs[iddb]) +
                                  beta * fs[idb]) / (1 + 4 * alpha + beta);
                    /* curvature.c:176 weights fs[idl]; the corrected option fs[idu] */
                    const int fixed = p->curvature_corrected != 0;
                    double fsu = (fs[idufl] + fs[idufr] + fs[idubr] + fs[idubl] +
                                  alpha * (fs[idul] + fs[idur] + fs[idub] + fs[iduf]) +
                                  beta * fs[fixed ? idu : idl]) / (1 + 4 * alpha + beta);
                    double fsd = (fs[iddbr] + fs[iddbl] + fs[iddfl] + fs[iddfr] +
                                  alpha * (fs[iddr] + fs[iddl] + fs[iddf] + fs[iddb]) +
                                  beta * fs[idd]) / (1 + 4 * alpha + beta);
                    double nx_ = (fsl - fsr) / 2.0, ny_ = (fsf - fsb) / 2.0, nz_ = (fsu - fsd) / 2.0;
                    double nall = sqrt(nx_ * nx_ + ny_ * ny_ + nz_ * nz_);
                    /* curvature.c:194 and 203 as written, or corrected */
                    if (fixed ? (nall != 0.0) : !(nall)) {
                        nx_ = nx_ / nall;
                        ny_ = ny_ / nall;
                        nz_ = nz_ / nall;
                    }
                    int nor_dir = 0;
                    if (fixed || !(nx_) || !(ny_) || !(nz_)) {
                        if ((fabs(nx_) >= fabs(ny_)) && (fabs(nx_) >= fabs(nz_))) nor_dir = 1;
                        else if ((fabs(ny_) >= fabs(nz_)) && (fabs(ny_) >= fabs(nx_))) nor_dir = 2;
                        else if ((fabs(nz_) >= fabs(ny_)) && (fabs(nz_) >= fabs(nx_))) nor_dir = 3;
                    }
                    double gamma, hx, hy, hxx, hyy, hxy;
                    int t;
                    long st; /* stride along the height direction */
                    long a1, a2, b1, b2, c11, c12, c21, c22;
                    double ncomp;
                    int pos, dim;
                    if (nor_dir == 3) {
                        ncomp = nz_; pos = k; dim = dimz; st = kgap;
                        /* h, hf, hb, hl, hr, hfl, hfr, hbr, hbl */
                        a1 = idf; a2 = idb; b1 = idl; b2 = idr;
                        c11 = idfl; c12 = idfr; c21 = idbl; c22 = idbr;
                    } else if (nor_dir == 2) {
                        ncomp = ny_; pos = j; dim = dimy; st = jgap;
                        /* h, hu, hd, hl, hr, hul, hur, hdr, hdl */
                        a1 = idu; a2 = idd; b1 = idl; b2 = idr;
                        c11 = idul; c12 = idur; c21 = iddl; c22 = iddr;
                    } else if (nor_dir == 1) {
                        ncomp = nx_; pos = i; dim = dimx; st = 1;
                        /* h, hu, hd, hf, hb, huf, hub, hdb, hdf */
                        a1 = idu; a2 = idd; b1 = idf; b2 = idb;
                        c11 = iduf; c12 = idub; c21 = iddf; c22 = iddb;
                    } else {
                        continue;
                    }
                    gamma = (acos(fabs(ncomp)) < 0.8) ? 0.0 : 0.2;
                    t = (((pos + 2) <= dim) && (pos - 2) >= 1) ? 3 : 1;
                    double h = 0, hA1 = 0, hA2 = 0, hB1 = 0, hB2 = 0, hC11 = 0, hC12 = 0, hC22 = 0, hC21 = 0;
                    for (int n = -t; n <= t; n++) {
                        h += fs[idx + st * n];
                        hA1 += fs[a1 + st * n];
                        hA2 += fs[a2 + st * n];
                        hB1 += fs[b1 + st * n];
                        hB2 += fs[b2 + st * n];
                        hC11 += fs[c11 + st * n];
                        hC12 += fs[c12 + st * n];
                        hC22 += fs[c22 + st * n];
                        hC21 += fs[c21 + st * n];
                    }
                    double cs = p->cellSize;
                    if (nor_dir == 3) {
                        /* hf=A1 hb=A2 hl=B1 hr=B2 hfl=C11 hfr=C12 hbl=C21 hbr=C22 */
                        hx = (gamma * (hC11 - hC12) + hB1 - hB2 + gamma * (hC21 - hC22)) / (1 + 2 * gamma) / 2.0;
                        hy = (gamma * (hC11 - hC21) + hA1 - hA2 + gamma * (hC12 - hC22)) / (1 + 2 * gamma) / 2.0;
                        hxx = (gamma * (hC11 - 2 * hA1 + hC12) + hB1 - 2 * h + hB2 +
                               gamma * (hC21 - 2 * hA2 + hC22)) / (cs) / (1 + 2 * gamma);
                        hyy = (gamma * (hC11 - 2 * hB1 + hC21) + hA1 - 2 * h + hA2 +
                               gamma * (hC12 - 2 * hB2 + hC22)) / (cs) / (1 + 2 * gamma);
                        hxy = (hC11 - hC21 - hC12 + hC22) / cs / 4.0;
                    } else if (nor_dir == 2) {
                        /* hu=A1 hd=A2 hl=B1 hr=B2 hul=C11 hur=C12 hdl=C21 hdr=C22 */
                        hx = (gamma * (hC11 - hC12) + hB1 - hB2 + gamma * (hC21 - hC22)) / (1 + 2 * gamma) / 2.0;
                        hy = (gamma * (hC11 - hC21) + hA1 - hA2 + gamma * (hC12 - hC22)) / (1 + 2 * gamma) / 2.0;
                        hxx = (gamma * (hC11 - 2 * hA1 + hC12) + hB1 - 2 * h + hB2 +
                               gamma * (hC21 - 2 * hA2 + hC22)) / (cs) / (1 + 2 * gamma);
                        hyy = (gamma * (hC11 - 2 * hB1 + hC21) + hA1 - 2 * h + hA2 +
                               gamma * (hC12 - 2 * hB2 + hC22)) / (cs) / (1 + 2 * gamma);
                        hxy = (hC11 - hC21 - hC12 + hC22) / cs / 4.0;
                    } else {
                        /* hu=A1 hd=A2 hf=B1 hb=B2 huf=C11 hub=C12 hdf=C21 hdb=C22 */
                        hx = (gamma * (hC11 - hC12) + hB1 - hB2 + gamma * (hC21 - hC22)) / (1 + 2 * gamma) / 2.0;
                        hy = (gamma * (hC11 - hC21) + hA1 - hA2 + gamma * (hC12 - hC22)) / (1 + 2 * gamma) / 2.0;
                        hxx = (gamma * (hC11 - 2 * hA1 + hC12) + hB1 - 2 * h + hB2 +
                               gamma * (hC21 - 2 * hA2 + hC22)) / (cs) / (1 + 2 * gamma);
                        hyy = (gamma * (hC11 - 2 * hB1 + hC21) + hA1 - 2 * h + hA2 +
                               gamma * (hC12 - 2 * hB2 + hC22)) / (cs) / (1 + 2 * gamma);
                        hxy = (hC11 - hC21 - hC12 + hC22) / cs / 4.0;
                    }
                    o->curv[idx] = (hxx + hyy + hxx * hy * hy + hyy * hx * hx - 2 * hxy * hx * hy) /
                                   pow((1 + hx * hx + hy * hy), 1.5);
                }
    }
}

/* fs_change_diffuse, growth.c:176-329 (!FSSEP branch 206-276) */
static void fs_change(mmso *o)
{
    const mms_params *p = &o->p;
    const double liq_slope = p->m_solute0;
    const double k_inv = 1.0 / p->part_coef;
    const double km = 1.0 - p->part_coef;
    const double km_inv = 1.0 / km;
    const double m_inv = 1.0 / liq_slope;
    const double D_x = p->Dliq / p->cellSize / p->cellSize;
    const double D_xt = D_x * p->ts_delt;
    const double cinit = p->Cinit;
    const double Tliq = p->liquidusTemp;
    double *ce = o->ce, *oce = o->oce, *fs = o->fs, *cl = o->cl;
    int *gr = o->gr;
    for (long k = 1; k <= o->gz; k++)
        for (long j = 1; j <= o->gy; j++)
            for (long i = 1; i <= o->gx; i++) {
                long idx = cidx(o, i, j, k);
                double Tcell = o->T[idx];
                double c_int = cinit + m_inv * (Tcell - Tliq);
                double Tunder = Tliq - Tcell;
                Tunder += liq_slope * (cl[idx] - cinit);
                if (gr[idx] <= 0 || Tcell < 1.0 || Tcell > Tliq) {
                    cl[idx] = ce[idx];
                    gr[idx] = 0;
                    fs[idx] = 0;
                    continue;
                }
                if (fs[idx] == 1.0 && (Tunder >= 0.0)) {
                    cl[idx] = ce[idx] * k_inv;
                    continue;
                }
                if (p->tip_curv) {
                    c_int = cinit + m_inv * (Tcell - Tliq + p->gibbs_coef * o->curv[idx]);
                    Tunder = Tliq - Tcell - p->gibbs_coef * o->curv[idx];
                }
                double dce = ce[idx] - oce[idx];
                double dcl = (c_int - cl[idx]) * D_xt * 2 + dce / (1 - km * fs[idx]);
                double dfs = (dcl * (1. - km * fs[idx]) - dce) * km_inv / cl[idx];
                cl[idx] += dcl;
                fs[idx] += dfs;
                fs[idx] = MINF(1.0, fs[idx]);
                if (fs[idx] < 0.) {
                    fs[idx] = 0.;
                    gr[idx] = 0;
                    cl[idx] = ce[idx];
                }
            }
}

/* grow_octahedra, growth.c:338-458 (!GROWSEP branch 357-407) */
static void grow(mmso *o)
{
    const mms_params *p = &o->p;
    const double fsgrow = p->rev_fsgrow;
    for (long k = 1; k <= o->gz; k++)
        for (long j = 1; j <= o->gy; j++)
            for (long i = 1; i <= o->gx; i++) {
                long idx = cidx(o, i, j, k);
                int grid = o->gr[idx];
                if (grid > 0 && (uint64_t)grid < p->maxTotalGrains) {
                    const double(*R)[3] = o->grains[grid].rotmat;
                    double g00 = R[0][0], g10 = R[1][0], g20 = R[2][0];
                    double g01 = R[0][1], g11 = R[1][1], g21 = R[2][1];
                    double g02 = R[0][2], g12 = R[1][2], g22 = R[2][2];
                    double rx0 = 0.0 - o->dc[idx].x;
                    double ry0 = 0.0 - o->dc[idx].y;
                    double rz0 = 0.0 - o->dc[idx].z;
                    double gx0 = g00 * rx0 + g10 * ry0 + g20 * rz0;
                    double gy0 = g01 * rx0 + g11 * ry0 + g21 * rz0;
                    double gz0 = g02 * rx0 + g12 * ry0 + g22 * rz0;
                    double ds1 = fabs(gx0) + fabs(gy0) + fabs(gz0);
                    ds1 = MINF(ds1, 1.5);
                    o->d[idx] = ds1 + o->fs[idx] * fsgrow;
                }
            }
}

/* grow_cell_reduction, growth.c:460-538, per rank in local raster order */
static void cell_reduction(mmso *o)
{
    const mms_params *p = &o->p;
    for (int r = 0; r < o->nranks; r++) {
        rank_t *rk = &o->ranks[r];
        long g = 0;
        for (long k = 1; k <= p->gsdimz; k++)
            for (long j = 1; j <= p->gsdimy; j++)
                for (long i = 1; i <= p->gsdimx; i++) {
                    long idx = rank_cell(o, rk, i, j, k);
                    if (o->mold[idx]) continue;
                    if (o->gr[idx] <= 0) {
                        int nbindex = o->gr[idx + 1] + o->gr[idx - 1] + o->gr[idx + o->sy] +
                                      o->gr[idx - o->sy] + o->gr[idx + o->sz] + o->gr[idx - o->sz];
                        if (nbindex > 0) rk->list[++g] = idx;
                    }
                }
        rk->gindex = g;
    }
}

/* capture_octahedra_diffuse, growth.c:573-808 (INDEX_SEP branch 640-808) */
static void capture(mmso *o)
{
    const mms_params *p = &o->p;
    static const short nn[6][3] = {{1, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    memcpy(o->ogr, o->gr, sizeof(int) * (size_t)o->N);
    const int *ogr = o->ogr;
    for (int r = 0; r < o->nranks; r++) {
        rank_t *rk = &o->ranks[r];
        long gindex = rk->gindex;
        if (gindex > rk->dc_tmp_size) {
            free(rk->dc_tmp);
            rk->dc_tmp_size = gindex + 100;
            rk->dc_tmp = (dc3 *)calloc((size_t)rk->dc_tmp_size, sizeof(dc3));
        }
        for (long i = 1; i <= gindex; i++) {
            long idx = rk->list[i];
            if (ogr[idx] > 0) continue;
            const long ndxs[6] = {idx + 1, idx + o->sy, idx - 1, idx - o->sy, idx + o->sz, idx - o->sz};
            double g00 = 0, g10 = 0, g20 = 0, g01 = 0, g11 = 0, g21 = 0, g02 = 0, g12 = 0, g22 = 0;
            double dx = 0, dy = 0, dz = 0;
            long ndx = 0;
            short found = -1;
            for (short n = 0; n < 6; n++) {
                ndx = ndxs[n];
                int gid = ogr[ndx];
                if (gid > 0 && (uint64_t)gid < p->maxTotalGrains) {
                    const double(*R)[3] = o->grains[gid].rotmat;
                    g00 = R[0][0]; g10 = R[1][0]; g20 = R[2][0];
                    g01 = R[0][1]; g11 = R[1][1]; g21 = R[2][1];
                    g02 = R[0][2]; g12 = R[1][2]; g22 = R[2][2];
                    double rx1 = -1.0 * nn[n][0] - o->dc[ndx].x;
                    double ry1 = -1.0 * nn[n][1] - o->dc[ndx].y;
                    double rz1 = -1.0 * nn[n][2] - o->dc[ndx].z;
                    dx = g00 * rx1 + g10 * ry1 + g20 * rz1;
                    dy = g01 * rx1 + g11 * ry1 + g21 * rz1;
                    dz = g02 * rx1 + g12 * ry1 + g22 * rz1;
                    double dfs = o->d[ndx] - (fabs(dx) + fabs(dy) + fabs(dz));
                    if (dfs > 0) {
                        found = n;
                        break;
                    }
                }
            }
            if (found > -1) {
                double ncx = 0., ncz = 0., ncy = 0.;
                double ncd = MINF(o->d[ndx], 1.0);
                double dd = o->d[ndx] - ncd;
                if (dx + dy >= 0 && dx - dy > 0 && dx + dz > 0 && dx - dz >= 0) ncx = dd;
                else if (dx + dy <= 0 && dx - dy < 0 && dx + dz < 0 && dx - dz <= 0) ncx = -1. * dd;
                else if (dy + dx > 0 && dy - dx >= 0 && dy + dz >= 0 && dy - dz > 0) ncy = dd;
                else if (dy + dx < 0 && dy - dx <= 0 && dy + dz <= 0 && dy - dz < 0) ncy = -1. * dd;
                else if (dz + dx >= 0 && dz - dx > 0 && dz + dy > 0 && dz - dy >= 0) ncz = dd;
                else ncz = -1. * dd;
                rk->dc_tmp[i].x = o->dc[ndx].x + nn[found][0] + g00 * ncx + g01 * ncy + g02 * ncz;
                rk->dc_tmp[i].y = o->dc[ndx].y + nn[found][1] + g10 * ncx + g11 * ncy + g12 * ncz;
                rk->dc_tmp[i].z = o->dc[ndx].z + nn[found][2] + g20 * ncx + g21 * ncy + g22 * ncz;
                o->gr[idx] = ogr[ndx];
                o->fs[idx] = 0.;
                o->cl[idx] = o->ce[idx];
            }
        }
        for (long i = 1; i <= gindex; i++) o->dc[rk->list[i]] = rk->dc_tmp[i];
    }
}

/* doiteration, calculate.c:192-352, preceded by loop.c:224 */
static int step_once(mmso *o)
{
    o->stepped = 1;
    o->timestep++;
    temp_update(o);
    nucleation(o);
    int st = activation(o);
    if (st) return st;
    memcpy(o->oce, o->ce, sizeof(double) * (size_t)o->N);
    st = diffuse(o);
    if (st) return st;
    if (o->curv_on && o->p.tip_curv) curvature(o);
    fs_change(o);
    grow(o);
    cell_reduction(o);
    capture(o);
    return MMS_OK;
}

int mmso_step(mmso *o, int nsteps)
{
    for (int s = 0; s < nsteps; s++) {
        int st = step_once(o);
        if (st) return st;
    }
    return MMS_OK;
}

uint64_t mmso_timestep(const mmso *o) { return o->timestep; }
int mmso_num_grains(const mmso *o) { return o->num_grains; }
size_t mmso_num_cells(const mmso *o) { return (size_t)o->N; }

int mmso_get_field(mmso *o, int field, void *out)
{
    size_t N = (size_t)o->N;
    switch (field) {
    case MMS_FIELD_CE: memcpy(out, o->ce, N * sizeof(double)); break;
    case MMS_FIELD_CL: memcpy(out, o->cl, N * sizeof(double)); break;
    case MMS_FIELD_FS: memcpy(out, o->fs, N * sizeof(double)); break;
    case MMS_FIELD_GR: memcpy(out, o->gr, N * sizeof(int)); break;
    case MMS_FIELD_DC: memcpy(out, o->dc, N * sizeof(dc3)); break;
    case MMS_FIELD_D: {
        /* grow_octahedra's value where the cell was solid at the growth step */
        double *dd = (double *)out;
        for (size_t c = 0; c < N; c++) dd[c] = o->ogr[c] > 0 ? o->d[c] : 0.0;
        break;
    }
    case MMS_FIELD_OGR: memcpy(out, o->ogr, N * sizeof(int)); break;
    case MMS_FIELD_NUC_THRESHOLD: memcpy(out, o->thr, N * sizeof(float)); break;
    case MMS_FIELD_TEMPERATURE: memcpy(out, o->T, N * sizeof(double)); break;
    case MMS_FIELD_MOLD: memcpy(out, o->mold, N); break;
    case MMS_FIELD_CURV: memcpy(out, o->curv, N * sizeof(double)); break;
    default: return MMS_ERR_ARG;
    }
    return MMS_OK;
}

/* reduce_fs per rank (growth.c:540-566), then the rank-ordered MPI_Reduce of
 * solid_volume (growth.c:971-978, loop.c:172-183) */
double mmso_reduce(mmso *o, int what)
{
    const mms_params *p = &o->p;
    if (what == MMS_REDUCE_CE_SUM) {
        double s = 0, c = 0;
        for (long k = 1; k <= o->gz; k++)
            for (long j = 1; j <= o->gy; j++)
                for (long i = 1; i <= o->gx; i++) {
                    double y = o->ce[cidx(o, i, j, k)] - c;
                    double t = s + y;
                    c = (t - s) - y;
                    s = t;
                }
        return s;
    }
    double svol = 0;
    for (int r = 0; r < o->nranks; r++) {
        rank_t *rk = &o->ranks[r];
        double sum_fs = 0.0;
        for (long k = 1; k <= p->gsdimz; k++)
            for (long j = 1; j <= p->gsdimy; j++)
                for (long i = 1; i <= p->gsdimx; i++) sum_fs += MINF(1.0, o->fs[rank_cell(o, rk, i, j, k)]);
        double v = sum_fs * pow(p->cellSize, 3.0);
        svol = (r == 0) ? v : svol + v;
    }
    if (what == MMS_REDUCE_SOLID_VOLUME) return svol;
    return svol / ((o->gx * o->gy * o->gz) * pow(p->cellSize, 3));
}

void mmso_get_grains(mmso *o, int first, int count, mms_grain *out)
{
    for (int i = 0; i < count; i++) {
        long g = first + i;
        if (g < o->grains_cap) out[i] = o->grains[g];
        else memset(&out[i], 0, sizeof(mms_grain));
    }
}

/* output_grains summary, grain.c:716-833 */
void mmso_grain_summary(mmso *o, mms_grain_summary *s)
{
    size_t *sizes = (size_t *)calloc((size_t)o->num_grains + 1, sizeof(size_t));
    for (long k = 1; k <= o->gz; k++)
        for (long j = 1; j <= o->gy; j++)
            for (long i = 1; i <= o->gx; i++) {
                int g = o->gr[cidx(o, i, j, k)];
                if (g > 0) sizes[g]++;
            }
    size_t minSize = sizes[1], maxSize = sizes[1], avgSize = 0, zeroCount = 0;
    double cellVolume = pow(o->p.cellSize * 1000, 3.0);
    for (int i = 1; i < o->num_grains; i++) {
        if (sizes[i] < minSize) minSize = sizes[i];
        if (sizes[i] > maxSize) maxSize = sizes[i];
        avgSize += sizes[i];
        if (sizes[i] == 0) zeroCount++;
    }
    s->num_grains = o->num_grains - 1;
    s->min_mm3 = minSize * cellVolume;
    s->max_mm3 = maxSize * cellVolume;
    s->avg_mm3 = ((double)avgSize / ((double)((o->num_grains - 1) - zeroCount)) * cellVolume);
    free(sizes);
}

/* loop, loop.c:185-271 (screen lines and checkDone, without data files) */
int mmso_run(mmso *o, int verbose)
{
    const mms_params *p = &o->p;
    int done = 0;
    double fs = 0.;
    if (verbose && p->screenpfreq > 0) {
        printf("\n%10s  %10s   %8s  %8s\n", "Wall Time", "Sim Time", "Fraction", "Grain NO");
        printf("%10s  %10s   %8s\n", "(sec)  ", "(sec)  ", "Solid");
    }
    while (!done) {
        int st = step_once(o);
        if (st) return st;
        if (p->screenpfreq > 0 && o->timestep % p->screenpfreq == 0) {
            fs = mmso_reduce(o, MMS_REDUCE_FS_FRACTION);
            if (verbose)
                printf("%10g  %10g  %8.4lf%% %8d  %s \n", 0.0, o->timestep * p->ts_delt, 100.0 * fs,
                       o->num_grains - 1, "\n");
        }
        if (p->finish_time && ((o->timestep * p->ts_delt) >= p->finish_time)) done = 1;
        if (fs >= p->fs_finish) done = 1;
    }
    if (verbose) {
        mms_grain_summary s;
        mmso_grain_summary(o, &s);
        printf("%d grains.  Min: %lg mm^3   Max: %lg mm^3   Average:  %lg mm^3\n", s.num_grains,
               s.min_mm3, s.max_mm3, s.avg_mm3);
    }
    return MMS_OK;
}

/* getRenumberArray (io_xdmf.c:344-375), called by the reference's XDMF
 * writer on rank 0 with RandomizeGrains: when the grain count has grown
 * since the last call, a fresh shuffle of ids 1..n-1 drawn from rank 0's
 * rand() stream, which its later orientation draws then follow.  Returns
 * the renumbering's length; up to cap entries go to out. */
int mmso_xdmf_renumber(mmso *o, uint64_t *out, int cap)
{
    const int ng = o->num_grains;
    if (!o->renum || ng > o->renum_n) {
        free(o->renum);
        o->renum = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)ng);
        for (int i = 0; i < ng; i++) o->renum[i] = (uint64_t)i;
        for (int i = 1; i < ng; i++) {
            int pic;
            do {
                pic = rng_rand(&o->ranks[0]) % ng;
            } while (pic == 0);
            uint64_t t = o->renum[pic];
            o->renum[pic] = o->renum[i];
            o->renum[i] = t;
        }
        o->renum_n = ng;
    }
    for (int i = 0; i < cap && i < o->renum_n; i++) out[i] = o->renum[i];
    return o->renum_n;
}
