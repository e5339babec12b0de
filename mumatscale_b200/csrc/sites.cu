// sites.cu — nucleation sites drawn on the device (mms_params.site_setup 1).
//
// init_sb_nucleation (grain.c:930-1010) picks, per rank, exactly
// floor(rho_v V dx^3) of its V non-mold cells (Knuth's Algorithm S on the
// rank's rand() stream, grain.c:250-296) and gives each a threshold drawn
// from N(centre, sigma), redrawn while below 1e-5 or more than 6 sigma off
// (genRandomThreshold, grain.c:140-154); then the same for surface sites
// among the cells next to the mold, skipping cells already chosen.  That
// replay is sequential host work over every cell.  Here each cell is
// chosen independently with the rank's probability count / V (so the site
// count is binomial around the reference's exact count), from a
// counter-based generator, Philox4x32-10 (Salmon, Moraes, Dror and Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), whose counter is
// the cell's position in (rank, local raster) order and whose key is
// RandSeedVal: any cell's draws are available in any order, so the site
// list comes out of two passes over the cells in list order with no dense
// intermediate arrays.  Deck-defined sites (FixedNuc, NucVolume) are given
// as presets and win over drawn ones, as the reference's select_if_not_fixed
// (grain.c:225-237) leaves them.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "mms_internal.h"
#include "sites.h"

namespace mms {
namespace {

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
    const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const unsigned hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        const unsigned hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += W0;
        k.y += W1;
    }
    return c;
}

// (0, 1]
__device__ __forceinline__ double unit(unsigned a, unsigned b)
{
    const unsigned long long v = ((unsigned long long)a << 21) ^ (unsigned long long)b;  // 53 bits
    return ((double)(v & ((1ULL << 53) - 1)) + 1.0) * (1.0 / 9007199254740992.0);
}

// threshold of cell q (list position in (rank, local raster) order), or +inf
__device__ float draw_cell(const SiteDrawArgs &a, const double *pv, const double *ps, const long long *pq,
                           const float *pt, long long q)
{
    const long long r = q / a.sbcells, l = q - r * a.sbcells;
    // a deck-defined site wins
    long long lo = 0, hi = a.npreset - 1;
    while (lo <= hi) {
        const long long mid = (lo + hi) >> 1;
        if (pq[mid] == q) return pt[mid];
        if (pq[mid] < q) lo = mid + 1;
        else hi = mid - 1;
    }
    const uint2 key = make_uint2(a.seed, 0x5EED5EEDu);
    uint4 c = make_uint4((unsigned)q, (unsigned)(q >> 32), 0u, 0u);
    const uint4 u = philox4x32_10(c, key);
    double centre, sigma;
    if (unit(u.x, u.y) <= pv[r]) {
        centre = a.vol_centre;
        sigma = a.vol_sigma;
    } else {
        // next to the mold: a pad face of the whole domain
        const int sbx = a.sbx, sby = a.sby;
        const long long lz = l / ((long long)sbx * sby), ly = (l / sbx) % sby, lx = l % sbx;
        const int rx = (int)(r % a.nsbx), ry = (int)((r / a.nsbx) % a.nsby), rz = (int)(r / ((long long)a.nsbx * a.nsby));
        const long long I = (long long)rx * sbx + lx + 1, J = (long long)ry * sby + ly + 1,
                        K = (long long)rz * a.sbz + lz + 1;
        const bool surf = (a.padx && (I == 1 || I == a.gx)) || (a.pady && (J == 1 || J == a.gy)) ||
                          (a.padz && (K == 1 || K == a.gz));
        if (!(surf && unit(u.z, u.w) <= ps[r])) return INFINITY;
        centre = a.surf_centre;
        sigma = a.surf_sigma;
    }
    // genRandomThreshold's rule, with a bound on the redraws (the chance of
    // a redraw is below 1e-8 for the decks' parameters)
    for (unsigned att = 1; att < 64; att++) {
        c.z = 1u;
        c.w = att;
        const uint4 v = philox4x32_10(c, key);
        const double z = sqrt(-2.0 * log(unit(v.x, v.y))) * cos(6.283185307179586 * unit(v.z, v.w));
        const float t = (float)(sigma * z + centre);
        if (!((t < 1.0e-5f) || (fabs((double)t - centre) > (6.0 * sigma)))) return t;
    }
    return (float)centre;
}

constexpr int SD_NT = 256, SD_PER = 16;

__global__ void __launch_bounds__(SD_NT) k_site_count(SiteDrawArgs a, const double *pv, const double *ps,
                                                      const long long *pq, const float *pt, int *blk_count)
{
    __shared__ int sh[SD_NT / 32];
    const long long l0 = ((long long)blockIdx.x * SD_NT + threadIdx.x) * SD_PER;
    int n = 0;
    for (int i = 0; i < SD_PER; i++) {
        const long long li = l0 + i;
        if (li < a.total && draw_cell(a, pv, ps, pq, pt, a.qbase + li) != INFINITY) n++;
    }
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < SD_NT / 32; w++) t += sh[w];
        blk_count[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(SD_NT) k_site_write(SiteDrawArgs a, const double *pv, const double *ps,
                                                      const long long *pq, const float *pt, const long long *blk_off,
                                                      long long *cell, float *thr, int *rank)
{
    __shared__ int sh[SD_NT / 32];
    const long long l0 = ((long long)blockIdx.x * SD_NT + threadIdx.x) * SD_PER;
    float t[SD_PER];
    int n = 0;
    for (int i = 0; i < SD_PER; i++) {
        const long long li = l0 + i;
        t[i] = (li < a.total) ? draw_cell(a, pv, ps, pq, pt, a.qbase + li) : INFINITY;
        n += t[i] != INFINITY;
    }
    // exclusive prefix of n over the block, in thread order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = n;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) sh[warp] = incl;
    __syncthreads();
    int base = 0;
    for (int w = 0; w < warp; w++) base += sh[w];
    long long pos = blk_off[blockIdx.x] + base + incl - n;
    for (int i = 0; i < SD_PER; i++) {
        if (t[i] == INFINITY) continue;
        const long long q = a.qbase + l0 + i;
        const long long r = q / a.sbcells, l = q - r * a.sbcells;
        const long long lz = l / ((long long)a.sbx * a.sby), ly = (l / a.sbx) % a.sby, lx = l % a.sbx;
        const int rx = (int)(r % a.nsbx), ry = (int)((r / a.nsbx) % a.nsby), rz = (int)(r / ((long long)a.nsbx * a.nsby));
        const long long I = (long long)rx * a.sbx + lx + 1, J = (long long)ry * a.sby + ly + 1,
                        K = (long long)rz * a.sbz + lz + 1 - a.kz0;
        cell[pos] = K * a.dsz + J * a.dsy + I;
        thr[pos] = t[i];
        rank[pos] = (int)r - a.rank0;
        pos++;
    }
}

}  // namespace

int site_draw_device(const SiteDrawArgs &args, const std::vector<double> &pv, const std::vector<double> &ps,
                     const std::vector<long long> &preset_q, const std::vector<float> &preset_thr,
                     std::vector<long long> &cells, std::vector<float> &thr, std::vector<int> &rank, std::string &err)
{
    SiteDrawArgs a = args;
    a.npreset = (long long)preset_q.size();
    const long long per_blk = (long long)SD_NT * SD_PER;
    const long long nblk = (a.total + per_blk - 1) / per_blk;
    cells.clear();
    thr.clear();
    rank.clear();
    if (a.total <= 0) return 0;
    double *dpv = nullptr, *dps = nullptr;
    long long *dpq = nullptr, *doff = nullptr, *dcell = nullptr;
    float *dpt = nullptr, *dthr = nullptr;
    int *dcnt = nullptr, *drank = nullptr;
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t x) {
        if (e == cudaSuccess && x != cudaSuccess) e = x;
        return e == cudaSuccess;
    };
    const size_t np = preset_q.size() ? preset_q.size() : 1;
    if (chk(cudaMalloc(&dpv, pv.size() * sizeof(double))) && chk(cudaMalloc(&dps, ps.size() * sizeof(double))) &&
        chk(cudaMalloc(&dpq, np * sizeof(long long))) && chk(cudaMalloc(&dpt, np * sizeof(float))) &&
        chk(cudaMalloc(&dcnt, (size_t)nblk * sizeof(int))) && chk(cudaMalloc(&doff, (size_t)nblk * sizeof(long long))) &&
        chk(cudaMemcpy(dpv, pv.data(), pv.size() * sizeof(double), cudaMemcpyHostToDevice)) &&
        chk(cudaMemcpy(dps, ps.data(), ps.size() * sizeof(double), cudaMemcpyHostToDevice)) &&
        (preset_q.empty() ||
         (chk(cudaMemcpy(dpq, preset_q.data(), preset_q.size() * sizeof(long long), cudaMemcpyHostToDevice)) &&
          chk(cudaMemcpy(dpt, preset_thr.data(), preset_thr.size() * sizeof(float), cudaMemcpyHostToDevice))))) {
        k_site_count<<<(unsigned)nblk, SD_NT>>>(a, dpv, dps, dpq, dpt, dcnt);
        std::vector<int> cnt((size_t)nblk);
        std::vector<long long> off((size_t)nblk);
        if (chk(cudaGetLastError()) && chk(cudaMemcpy(cnt.data(), dcnt, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost))) {
            long long tot = 0;
            for (long long b = 0; b < nblk; b++) off[b] = tot, tot += cnt[b];
            const size_t nt = tot ? (size_t)tot : 1;
            if (chk(cudaMemcpy(doff, off.data(), off.size() * sizeof(long long), cudaMemcpyHostToDevice)) &&
                chk(cudaMalloc(&dcell, nt * sizeof(long long))) && chk(cudaMalloc(&dthr, nt * sizeof(float))) &&
                chk(cudaMalloc(&drank, nt * sizeof(int)))) {
                k_site_write<<<(unsigned)nblk, SD_NT>>>(a, dpv, dps, dpq, dpt, doff, dcell, dthr, drank);
                cells.resize((size_t)tot);
                thr.resize((size_t)tot);
                rank.resize((size_t)tot);
                chk(cudaGetLastError()) &&
                    chk(cudaMemcpy(cells.data(), dcell, (size_t)tot * sizeof(long long), cudaMemcpyDeviceToHost)) &&
                    chk(cudaMemcpy(thr.data(), dthr, (size_t)tot * sizeof(float), cudaMemcpyDeviceToHost)) &&
                    chk(cudaMemcpy(rank.data(), drank, (size_t)tot * sizeof(int), cudaMemcpyDeviceToHost));
            }
        }
    }
    for (void *p : {(void *)dpv, (void *)dps, (void *)dpq, (void *)dpt, (void *)dcnt, (void *)doff, (void *)dcell,
                    (void *)dthr, (void *)drank})
        if (p) cudaFree(p);
    if (e != cudaSuccess) {
        err = std::string("device site draw: ") + cudaGetErrorString(e);
        return 1;
    }
    return 0;
}

}  // namespace mms
