// host_setup.cpp — the reference's site pre-draw replayed on the host.
// See host_setup.h.  Compiled as plain host C++ (no FMA contraction on
// x86-64), so every draw and threshold is bit-identical to the reference.
#include "host_setup.h"

#include <algorithm>
#include <cstdio>

namespace mms {

void Rank::seed_with(unsigned s)
{
    std::memset(&rd, 0, sizeof rd);
    std::memset(state, 0, sizeof state);
    initstate_r(s, state, sizeof state, &rd);
    seed = s;
    ncalls = 0;
    have_gauss = 0;
    gauss_next = 0.f;
}
namespace {
// rd's pointers re-expressed against another copy of the state buffer
void rebase(struct random_data &rd, const char *from, char *to)
{
    auto mv = [&](int32_t *q) { return q ? (int32_t *)(to + ((const char *)q - from)) : nullptr; };
    rd.fptr = mv(rd.fptr);
    rd.rptr = mv(rd.rptr);
    rd.state = mv(rd.state);
    rd.end_ptr = mv(rd.end_ptr);
}
}  // namespace

void Rank::save(RngState &out) const
{
    std::memcpy(out.state, state, sizeof state);
    out.rd = rd;
    rebase(out.rd, state, out.state);
    out.ncalls = ncalls;
    out.have_gauss = have_gauss;
    out.gauss_next = gauss_next;
}

void Rank::restore(const RngState &in)
{
    std::memcpy(state, in.state, sizeof state);
    rd = in.rd;
    rebase(rd, in.state, state);
    ncalls = in.ncalls;
    have_gauss = in.have_gauss;
    gauss_next = in.gauss_next;
}

int32_t Rank::rand_()
{
    int32_t v;
    random_r(&rd, &v);
    ncalls++;
    return v;
}
// getRandScale, functions.c:440-445
float Rank::scale() { return (float)rand_() / (float)RAND_MAX; }
// getRandomGaussian, functions.c:376-406 (log of the float s is taken in
// double, as C's argument promotion does in the reference)
float Rank::gauss()
{
    if (have_gauss) {
        have_gauss = 0;
        return gauss_next;
    }
    float n0, n1, s;
    do {
        n0 = ((float)rand_() / (float)(RAND_MAX / 2.0)) - 1.0;
        n1 = ((float)rand_() / (float)(RAND_MAX / 2.0)) - 1.0;
        s = n0 * n0 + n1 * n1;
    } while (s >= 1.0 || s == 0);
    float multiplier = sqrtf(-2.0 * ::log((double)s) / s);
    float val = n0 * multiplier;
    gauss_next = n1 * multiplier;
    have_gauss = 1;
    return val;
}

// nucleate_grain's rotation matrix (grain.c:314-336), row-major
void rotmat_from_angles(double a0, double a1, double a2, double *R)
{
    double c0 = cos(a0), s0 = sin(a0), c1 = cos(a1), s1 = sin(a1), c2 = cos(a2), s2 = sin(a2);
    R[0] = c2 * c0 - s2 * s1 * s0;          // [0][0]
    R[3] = c2 * s0 + s2 * c1 * c0;          // [1][0]
    R[6] = s2 * s1;                         // [2][0]
    R[1] = -1. * s2 * c0 - c2 * c1 * s0;    // [0][1]
    R[4] = -1. * s2 * s0 + c2 * c1 * c0;    // [1][1]
    R[7] = c2 * s1;                         // [2][1]
    R[2] = s1 * s0;                         // [0][2]
    R[5] = -1. * s1 * c0;                   // [1][2]
    R[8] = c1;                              // [2][2]
}


namespace {
// host arrays of the setup use the reference layout
long long cidx(const Geo &g, long long i, long long j, long long k) { return ref_index(g, i, j, k); }
}  // namespace

// realcoord2scoord, functions.c:91-107
void real2cell(const mms_params &p, double x, double y, double z, size_t *i, size_t *j, size_t *k)
{
    x = x - p.origin_offset[0] + p.cellSize * 0.1;
    y = y - p.origin_offset[1] + p.cellSize * 0.1;
    z = z - p.origin_offset[2] + p.cellSize * 0.1;
    *i = (size_t)(x / p.cellSize);
    *j = (size_t)(y / p.cellSize);
    *k = (size_t)(z / p.cellSize);
}

// CELLCOORD2REALCOORDn, functions.h:284-286
double cell2real(const mms_params &p, int axis, double i) { return p.origin_offset[axis] + (i + 0.5) * p.cellSize; }

int rank_of_cell(const mms_params &p, size_t cx, size_t cy, size_t cz)
{
    long x = (long)(cx / (size_t)p.gsdimx), y = (long)(cy / (size_t)p.gsdimy), z = (long)(cz / (size_t)p.gsdimz);
    if (!p.padBndyX) x = (x + p.gnsbx) % p.gnsbx;
    if (!p.padBndyY) y = (y + p.gnsby) % p.gnsby;
    if (!p.padBndyZ) z = (z + p.gnsbz) % p.gnsbz;
    if (x < 0 || y < 0 || z < 0 || x >= p.gnsbx || y >= p.gnsby || z >= p.gnsbz) return -1;
    return (int)(x + y * p.gnsbx + z * p.gnsbx * p.gnsby);
}

// setNucOrientation, grain.c:117-130
void draw_orientation(const mms_params &p, Rank &r, NucPt &n)
{
    n.gx = n.gy = n.gz = 0.0;
    if (p.gnUseOrientation) {
        float acon = 4.0;
        n.gx = M_PI / acon - 2 * (M_PI / acon * r.scale());
        n.gy = M_PI / acon - 2 * (M_PI / acon * r.scale());
        n.gz = M_PI / acon - 2 * (M_PI / acon * r.scale());
    }
}

// distribute_nucleations (Knuth Algorithm S), grain.c:250-296
template <typename F>
void algorithm_s(Rank &r, size_t nc, size_t num, F select)
{
    size_t n = std::min(num, nc);
    size_t N = nc, t = 0, m = 0, idx = 0;
    if (n == 0) return;
    do {
        double U = r.scale();
        if ((N - t) * U >= (n - m)) {
            t++;
        } else {
            select(idx);
            t++;
            m++;
        }
        idx++;
    } while (m < n);
}

// genRandomThreshold, grain.c:140-154
float random_threshold(Rank &r, double center, double sigma)
{
    float t = 0.0;
    do {
        t = (float)(sigma * r.gauss() + center);
    } while ((t < 1.0e-5) || (fabs(t - center) > (6.0 * sigma)));
    return t;
}

// Host-side initial state: SetupInitialConditions (setup.c:41-94),
// init_nucleation_sites (grain.c:602-713, rank 0) and init_sb_nucleation
// (grain.c:930-1010, every rank).  Produces the dense threshold array.
void assign_deck_sites(const mms_params &p, const Geo &g, const std::vector<mms_fixed_nuc> &fixed,
                       const std::vector<mms_nuc_volume> &vols, std::vector<Rank> &ranks)
{
    Rank &r0 = ranks[0];
    std::vector<NucPt> all;
    for (const mms_fixed_nuc &f : fixed) {
        NucPt n{};
        n.x = f.x;
        n.y = f.y;
        n.z = f.z;
        n.gx = (M_PI / 180.0) * f.ax;
        n.gy = (M_PI / 180.0) * f.ay;
        n.gz = (M_PI / 180.0) * f.az;
        n.threshold = f.threshold;
        real2cell(p, n.x, n.y, n.z, &n.cx, &n.cy, &n.cz);
        all.push_back(n);
    }
    for (mms_nuc_volume v : vols) {
        v.minx = std::max(v.minx, p.origin_offset[0]);
        v.maxx = std::min(v.maxx, p.origin_offset[0] + (g.gx * p.cellSize));
        v.miny = std::max(v.miny, p.origin_offset[1]);
        v.maxy = std::min(v.maxy, p.origin_offset[1] + (g.gy * p.cellSize));
        v.minz = std::max(v.minz, p.origin_offset[2]);
        v.maxz = std::min(v.maxz, p.origin_offset[2] + (g.gz * p.cellSize));
        size_t mn[3], mx[3];
        real2cell(p, v.minx, v.miny, v.minz, &mn[0], &mn[1], &mn[2]);
        real2cell(p, v.maxx, v.maxy, v.maxz, &mx[0], &mx[1], &mx[2]);
        size_t count = (mx[0] - mn[0]) * (mx[1] - mn[1]) * (mx[2] - mn[2]);
        size_t max_nucs = count * v.density;
        size_t nx = mx[0] - mn[0], ny = mx[1] - mn[1];
        algorithm_s(r0, count, max_nucs, [&](size_t index) {  // select_nuc_volume, grain.c:173-210
            NucPt n{};
            n.cx = mn[0] + index % nx;
            n.cy = mn[1] + (index % (nx * ny)) / nx;
            n.cz = mn[2] + index / (nx * ny);
            n.threshold = v.threshold;
            draw_orientation(p, r0, n);
            n.x = cell2real(p, 0, (double)n.cx);
            n.y = cell2real(p, 1, (double)n.cy);
            n.z = cell2real(p, 2, (double)n.cz);
            all.push_back(n);
        });
    }
    for (const NucPt &n : all) {
        size_t cx, cy, cz;
        real2cell(p, n.x, n.y, n.z, &cx, &cy, &cz);
        int sb = rank_of_cell(p, cx, cy, cz);
        if (sb >= 0) ranks[sb].nuc.push_back(n);
    }
}

void setup_sites(const mms_params &p, const Geo &g, const std::vector<mms_fixed_nuc> &fixed,
                 const std::vector<mms_nuc_volume> &vols, std::vector<Rank> &ranks, std::vector<float> &thr,
                 const std::vector<signed char> &mold)
{
    assign_deck_sites(p, g, fixed, vols, ranks);
    // init_sb_nucleation per rank
    const long long sbcells = g.sbcells;
    std::vector<long long> vol, suf;
    vol.reserve(sbcells);
    suf.reserve(sbcells);
    for (int ri = 0; ri < g.nranks; ri++) {
        Rank &r = ranks[ri];
        r.ncalls_presb = r.ncalls;
        auto rcell = [&](long long i, long long j, long long k) {
            return cidx(g, (long long)r.sbx * p.gsdimx + i, (long long)r.sby * p.gsdimy + j,
                        (long long)r.sbz * p.gsdimz + k);
        };
        for (const NucPt &n : r.nuc) {
            long long c = rcell(1 + (long long)(n.cx % (size_t)p.gsdimx), 1 + (long long)(n.cy % (size_t)p.gsdimy),
                                1 + (long long)(n.cz % (size_t)p.gsdimz));
            if (!mold[c]) thr[c] = (float)n.threshold;
        }
        vol.clear();
        suf.clear();
        for (long long z = 1; z <= p.gsdimz; z++)
            for (long long y = 1; y <= p.gsdimy; y++)
                for (long long x = 1; x <= p.gsdimx; x++) {
                    long long c = rcell(x, y, z);
                    if (!mold[c]) {
                        vol.push_back(c);
                        int surf = mold[c - 1] + mold[c + 1] + mold[c - g.rsy] + mold[c + g.rsy] +
                                   mold[c - g.rsz] + mold[c + g.rsz];
                        if (surf) suf.push_back(c);
                    }
                }
        size_t v = vol.size(), s = suf.size();
        double center = p.gnGaussCenter, sigma = p.gnGaussSigma;
        auto sel = [&](const std::vector<long long> &cells) {
            return [&, cells_ptr = &cells](size_t index) {  // select_if_not_fixed, grain.c:225-237
                long long c = (*cells_ptr)[index];
                if (thr[c] == INFINITY) thr[c] = random_threshold(r, center, sigma);
            };
        };
        size_t count = p.maxGrainDensity * (v * pow(p.cellSize, 3.0));
        algorithm_s(r, v, count, sel(vol));
        if (p.doSurfaceNuc && (p.maxGrainDensitySurf > 0.0)) {
            center = p.gnGaussCenterSurf;
            sigma = p.gnGaussSigmaSurf;
            count = p.maxGrainDensitySurf * (s * pow(p.cellSize, 2.0));
            algorithm_s(r, s, count, sel(suf));
        }
    }
}


Geo make_geo(const mms_params &p)
{
    Geo g{};
    g.gx = p.gnsbx * p.gsdimx;
    g.gy = p.gnsby * p.gsdimy;
    g.gz = p.gnsbz * p.gsdimz;
    g.rsy = g.gx + 2;
    g.rsz = (long long)(g.gx + 2) * (g.gy + 2);
    g.rN = g.rsz * (g.gz + 2);
    // rows of the halo'd x extent plus the 3-element lead the stencil's tensor
    // maps start with (kernels.cu, alignment note), a multiple of 8 elements
    g.P = (g.gx + 2 + 3 + 7) / 8 * 8;
    g.sy = g.P;
    g.sz = g.P * (g.gy + 2);
    g.N = g.sz * (g.gz + 2);
    g.wpr = (g.gx + 31) / 32;
    g.nwords = (long long)g.wpr * (g.gy + 2) * (g.gz + 2);
    g.sbx = p.gsdimx;
    g.sby = p.gsdimy;
    g.sbz = p.gsdimz;
    g.nsbx = p.gnsbx;
    g.nsby = p.gnsby;
    g.nsbz = p.gnsbz;
    g.nranks = p.gnsbx * p.gnsby * p.gnsbz;
    g.sbcells = (long long)p.gsdimx * p.gsdimy * p.gsdimz;
    g.padx = p.padBndyX;
    g.pady = p.padBndyY;
    g.padz_lo = g.padz_hi = p.padBndyZ;
    g.ppr = (p.gsdimx + 31) / 32;
    g.pieces_per_rank = (long long)p.gsdimy * p.gsdimz * g.ppr;
    g.blocks_per_rank = (g.pieces_per_rank + LIST_PIECES - 1) / LIST_PIECES;
    g.ppr_m = div_magic((unsigned)g.ppr);
    g.sby_m = div_magic((unsigned)g.sby);
    return g;
}

std::vector<signed char> make_mold(const Geo &g)
{
    std::vector<signed char> mold((size_t)g.rN, 0);
    for (long long K = 0; K < g.gz + 2; K++)
        for (long long J = 0; J < g.gy + 2; J++)
            for (long long I = 0; I < g.gx + 2; I++) {
                int m = 0;
                if (g.padx && (I == 0 || I == g.gx + 1)) m = 1;
                if (g.pady && (J == 0 || J == g.gy + 1)) m = 1;
                if ((g.padz_lo && K == 0) || (g.padz_hi && K == g.gz + 1)) m = 1;
                mold[(size_t)cidx(g, I, J, K)] = (signed char)m;
            }
    return mold;
}

void init_ranks(const mms_params &p, const Geo &g, std::vector<Rank> &ranks)
{
    ranks.clear();
    ranks.resize(g.nranks);
    for (int r = 0; r < g.nranks; r++) {
        Rank &rk = ranks[r];
        rk.sbx = r % p.gnsbx;
        rk.sby = (r / p.gnsbx) % p.gnsby;
        rk.sbz = r / (p.gnsbx * p.gnsby);
        rk.seed_with((unsigned)r + 1 + p.base_random_seed);
    }
}

}  // namespace mms

// Site pre-draw without a device: the reference's nuc_threshold field after
// setup (setup.c:41-94, grain.c:602-713, 930-1010), in the halo'd layout.
extern "C" mms_status mms_predraw_sites(const mms_params *p, float *thr_out)
{
    using namespace mms;
    if (!p || !thr_out || p->gnsbx < 1 || p->gnsby < 1 || p->gnsbz < 1 || p->gsdimx < 1 || p->gsdimy < 1 ||
        p->gsdimz < 1 || p->cellSize <= 0)
        return MMS_ERR_ARG;
    Geo g = make_geo(*p);
    std::vector<Rank> ranks;
    init_ranks(*p, g, ranks);
    std::vector<signed char> mold = make_mold(g);
    std::vector<float> thr((size_t)g.rN, INFINITY);
    std::vector<mms_fixed_nuc> fixed(p->fixed_nucs, p->fixed_nucs + p->n_fixed_nucs);
    std::vector<mms_nuc_volume> vols(p->nuc_volumes, p->nuc_volumes + p->n_nuc_volumes);
    setup_sites(*p, g, fixed, vols, ranks, thr, mold);
    std::copy(thr.begin(), thr.end(), thr_out);
    return MMS_OK;
}
