// mms_internal.h — device-state layout shared by the host side (mms_api.cu)
// and the sm_100a kernels (kernels.cu).  Not part of the public ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mms.h"

extern "C" size_t mms_params_size(void);

namespace mms {

// Octahedron centre offset (decentered_t, globals.h:141-144).
struct Dc3 {
    double x, y, z;
};

// Device control block: everything a step needs that changes between steps
// lives here, so that a whole step (or a CUDA graph of many steps) runs with
// no host involvement.
struct Ctl {
    unsigned long long timestep;  // bp->timestep after the last committed step
    int num_grains;               // bp->num_grains (includes grain 0)
    int ncand;                    // nucleation candidates found this step
    int status;                   // first error (mms_status), 0 = ok
    int stall;                    // non-zero: later kernels of the step do nothing
    unsigned long long stall_step;
    int list_total;               // interface-list length over all ranks this step
    int list_ticket;              // k_list blocks started this step
    int new_grains;               // grains created by the last activation
    int rng_used_max;             // the most draws any rank consumed since the last refill
    // failure-detection test hook (mms_test_hold_list_block): k + 1 = the
    // interface-list block at position k publishes no status word, so the
    // look-back of the block after it waits for a word nothing writes; 0 =
    // none.  wait_polls: poll bound of the look-back waits (0 = about a
    // second, 2^22 polls)
    int hold_list_block;
    unsigned wait_polls;
    int nuc_done;                 // k_nuc_act blocks finished this step (the last one activates)
    int pad_;
};

enum StallReason : int {
    STALL_NONE = 0,
    STALL_ERROR = 1,      // ctl->status holds the error
    STALL_RNG = 2         // a rank ran out of pre-drawn orientations
};

// One record per created grain (index = grain id), enough for the host to
// rebuild grain_t (globals.h:244-254) for output_grains and mms_get_grains.
struct GrainLog {
    long long cell;       // device index of the nucleus cell; for a grain made by
                          // another slab (kind | GL_REMOTE), its reference-layout
                          // index in the whole domain
    unsigned long long timestep;
    int kind;             // 0 = deck site (nuc_pt entry), 1 = random draw, 2 = zero angles,
                          // 3 = pre-filled grain (mms_set_grains)
    int rank;             // emulated rank that created it (numbered over the whole domain)
    long long aux;        // nuc_pt entry index, or per-rank draw number
    float thr;            // nucleation threshold of the site
    int pad;
};
constexpr int GL_REMOTE = 8;

// A new grain as one slab publishes it to the others (z-slab split of one
// domain over several devices): its rotation and its record.
struct SlabRow {
    double rot[9];
    GrainLog lg;
};

// Geometry and physics constants passed to every kernel by value.
// Two layouts of the same halo'd grid: the reference's (row length gx+2,
// used by every host buffer crossing the ABI) and the device's, whose rows
// are padded to a multiple of 8 elements so that every row starts 64-byte
// aligned (TMA needs 16-byte strides).  Padding columns are never read.
struct Geo {
    int gx, gy, gz;            // interior cells
    long long P;               // device row pitch in elements (>= gx+2)
    long long sy, sz, N;       // device strides and size (sy = P)
    long long rsy, rsz, rN;    // reference layout strides and size (rsy = gx+2)
    int sbx, sby, sbz;         // NCellsPerSB
    int nsbx, nsby, nsbz;      // NSubblocks
    int nranks;
    long long sbcells;         // cells per subblock
    int padx, pady;            // pad (mold) faces
    int padz_lo, padz_hi;      // z faces: pad, or (0) a neighbouring slab's plane
    // bitmasks: one bit per interior cell, rows of wpr 32-bit words,
    // bit b of word w in row (j,k) = cell i = 1 + 32 w + b
    int wpr;
    long long nwords;          // wpr * (gy+2) * (gz+2)
    // interface-list pieces: 32 consecutive cells of one emulated rank's
    // local row; blocks of LIST_PIECES pieces in rank-local raster order
    int ppr;                   // pieces per local row = ceil(sbx / 32)
    long long pieces_per_rank; // sby * sbz * ppr
    long long blocks_per_rank; // ceil(pieces_per_rank / LIST_PIECES)
    // floor(2^32 / d) for d = ppr and d = sby (0xffffffff for d = 1): the
    // quotient of a 32-bit q by d is __umulhi(q, m) or one more
    unsigned ppr_m, sby_m;
};

inline unsigned div_magic(unsigned d) { return d <= 1 ? 0xffffffffu : (unsigned)((1ULL << 32) / d); }

constexpr int LIST_PIECES = 512;

inline long long dev_index(const Geo &g, long long i, long long j, long long k) { return k * g.sz + j * g.sy + i; }
inline long long ref_index(const Geo &g, long long i, long long j, long long k) { return k * g.rsz + j * g.rsy + i; }
inline long long ref_to_dev(const Geo &g, long long c)
{
    long long k = c / g.rsz, j = (c % g.rsz) / g.rsy, i = c % g.rsy;
    return dev_index(g, i, j, k);
}
inline long long dev_to_ref(const Geo &g, long long c)
{
    long long k = c / g.sz, j = (c % g.sz) / g.sy, i = c % g.sy;
    return ref_index(g, i, j, k);
}

struct Phys {
    // diffusion (growth.c:38-40)
    double rs, rl;
    // fs change (growth.c:181-197)
    double liq_slope, k_inv, km, km_inv, m_inv, D_xt, cinit, Tliq, Tsol;
    int tip_curv;
    int curv_fixed;  // mms_params.curvature_corrected
    double gibbs;
    // growth (growth.c:348)
    double fsgrow;
    unsigned long long max_grains;
    // nucleation (grain.c:1054-1059)
    double ma, mb, mc;
    // temperature (temperature.c:24-126)
    int temp_mode;   // 0 isothermal, 1 linear, 2 AM quadrature (array)
    double T0, cool_rate, gradient, grad_coef, velocity, velo_coef, ts_delt, cellSize;
    double origin[3];
    int gz_is_one;
    int kz0;         // global z of interior plane 1 minus 1 (a slab's offset; 0 for a whole domain)
    int am, amlayer;
    int use_orientation;
    double cellSize3;
};

// Everything device-resident for one context.
template <typename Real>
struct Fields {
    Real *ce;
    Real *cl[2];
    Real *fs[2];
};

struct DevPtrs {
    void *ce;
    void *cl[2];
    void *fs[2];
    int *gr;
    Dc3 *dc;
    unsigned *solid_bits;  // gr > 0 after fs_change (written by the stencil)
    double *T;            // AM temperature at the current step (N), FP64 form, or null
    float *T32;           // the same in the FP32 form (N), or null
    double *am_tab;       // AM quadrature tables (400 x (gx+gy+gz+6)) and plane flags
    float *am_ximg;       // FP32 form: the X table split into TF32 head and remainder in the
                          // tensor core's operand layout, then the Y and Z tables with the
                          // nodes contiguous (am_tc.cu), or null
    int *lsindex;         // AM layer flag or null
    double *curv;         // curvature (N) when TipCurvature
    // nucleation sites, sorted by (emulated rank, local raster)
    long long nsites;
    long long *site_cell;
    float *site_thr;
    int *site_rank;
    unsigned char *site_flag;
    int *cand;            // ordered candidate sites of the current step
    int *cand_stage;      // per nucleation block, its candidates in site order
    int *cand_ex;         // per candidate: random orientation draws before it (k_act)
    int *nuc_blk_cnt;     // candidates per nucleation block
    int nuc_blocks;
    // orientation sources
    long long n_nucpt;
    long long *nucpt_key;   // sorted global cell keys (first entry wins)
    long long *nucpt_entry; // index into the rank's nuc_pt list (host side)
    double *nucpt_rot;      // 9 per entry
    long long n_inj;
    long long *inj_key;
    double *inj_rot;
    double *rng_rot;        // nranks x rng_cap x 9
    int rng_cap;
    int *rng_used;          // per rank, draws consumed since rng_base
    long long *rng_base;    // per rank, absolute draw number of table entry 0
    int *act_scratch;       // 4 x nranks ints for k_act
    double zero_rot[9];     // rotation for zero angles (GNOriented 0)
    // grain table
    double *grain_rot;      // (max_grains + 1) x 9
    GrainLog *grain_log;    // (max_grains + 2)
    // interface list and capture
    unsigned long long *list_status;  // per list block: look-back status word
    int *blk_off;           // per list block: list position of its first entry
    int *rank_gindex;       // per rank, list length
    int *rank_dcsize;       // per rank, dc_tmp logical size
    int *rank_zero_upto;    // per rank: slots 1..n read as zero this step (0 = none)
    long long *rank_dcbase; // per rank, offset of its dc_tmp region
    long long *list_cell;   // list position -> cell
    int *list_gid;          // list position -> captured grain id (0 = not captured)
    Dc3 *dc_tmp;            // per-rank regions, 1-based slots
    // reductions
    double *red;            // scratch for partial sums
    double *fs_part;        // per stencil tile: (sum of the new fs, 0), then the folded total
    Ctl *ctl;
    // z-slab split of one domain (nslabs > 1): this slab's index, the
    // whole-domain number of its first emulated rank, the capacity of its
    // grain-row buffer; x1: per slab {candidates, short of draws} gathered
    // before activation; x2: per slab its new grains, gathered after it
    int nslabs, slab, rank0, slab_cap;
    int *x1_send;           // 2
    int *x1_recv;           // 2 x nslabs
    SlabRow *x2_send;       // slab_cap
    SlabRow *x2_recv;       // nslabs x slab_cap
    // frozen-CA record for the adjoint (null when not recording): per step
    // slot s (timestep rec_t0 + 1 + s), the fs_change branch of every cell
    // and, with TipCurvature, the curvature it used
    unsigned char *rec_flags;
    double *rec_curv;
    unsigned long long rec_t0;
    long long rec_cap;
};

// fs_change_diffuse branches (growth.c:228-272), as recorded for the adjoint
enum Branch : int {
    BR_RESET = 0,  // liquid / out of range: cl = ce, fs = 0
    BR_KEEP = 1,   // fully solid below liquidus: cl = ce / k
    BR_GROW = 2,   // growth update
    BR_CLAMP = 3,  // growth update with fs clamped to 1
    BR_NEG = 4     // growth update gave fs < 0: cl = ce, fs = 0
};

struct KernelArgs {
    Geo g;
    Phys p;
    DevPtrs d;
};

// Kernel ids for per-kernel timing.
enum KernelId : int {
    KID_TEMP_AM = 0, KID_NUC, KID_ACT, KID_CURV, KID_DIFFUSE_FS, KID_LIST, KID_CAPTURE, KID_COUNT
};

// Opaque storage for the stencil's TMA descriptors (built in kernels.cu).
struct TmaHolder {
    alignas(128) unsigned char bytes[6 * 128];
    int ok;
    int cpt = 1;  // stencil tile: cells per thread along x (1 or 2)
    int zc = 0;   // stencil z-chunk (0: chosen from the grid size)
};

// Optional event bracketing of each launch (mms_set_profiling).
struct Profiler {
    virtual void begin(int kid, void *stream) = 0;
    virtual void end(int kid, void *stream) = 0;
    virtual ~Profiler() {}
};

// Launchers implemented in kernels.cu.  Each returns the number of kernels
// it launched.
// start_stage 0: whole step; 1: resume at grain activation (after a stall).
// sumfs: the TMA stencil also leaves its per-tile fraction-solid sums in
// a.d.fs_part (see stencil_parts).
int launch_step(const KernelArgs &a, const TmaHolder &tma, int precision, void *stream, int start_stage,
                Profiler *prof, bool sumfs = false);
// Builds the TMA descriptors of the stencil for the current buffers;
// returns 0 when the driver cannot encode them (the stencil then uses its
// plain-load variant).
int make_tma(const KernelArgs &a, int precision, TmaHolder &out);
// the diffusion + fs-change stencil alone (tile autotuning)
int launch_stencil(const KernelArgs &a, const TmaHolder &tma, int precision, void *stream);
// the kernels of a step before / after the stencil
int launch_step_pre(const KernelArgs &a, int precision, void *stream, int start_stage);
int launch_step_post(const KernelArgs &a, int precision, void *stream);
int launch_curv(const KernelArgs &a, int precision, void *stream);
// One slab of a z-slab split, in three parts around the two exchanges of a
// step: phase 0 nucleation and the local half of activation (resume: only
// the latter), phase 1 grain ids and the stencil, phase 2 the other slabs'
// new grains, interface list and capture.
int launch_slab_phase(const KernelArgs &a, const TmaHolder &tma, int precision, void *stream, int phase,
                      int resume);
// Batched stencil over many domains: one item per domain (opaque, built by
// fill_batch_item, which returns the domain's tile count), one persistent
// launch of batch_grid CTAs.
size_t batch_item_bytes();
long long fill_batch_item(void *dst, const KernelArgs &a, const TmaHolder &tma, long long tile_begin);
int batch_grid(int precision, int cpt);
int launch_stencil_batch(const void *items, int nitems, long long total_tiles, int precision, int cpt, int grid,
                         void *stream);
// The other kernels of a step over all domains, one launch each: which = 0
// nucleation, 1 activation, 2 interface list, 3 capture; begin: device
// prefix sums (n + 1) of batch_blocks over the domains, total = begin[n].
int batch_blocks(const KernelArgs &a, int which);
int launch_small_batch(int which, const void *items, const int *begin, int n, int total, int precision,
                       void *stream);
// AM laser parameters (BB_struct, read_ctrl.c) for the moving-source quadrature
struct AmParams {
    double lsd, lv, lhs, lab, lpow, liniT, lthcon, rho_cp, x0, y0, z0;
    int amtracks, nsbx_times_sbx;
};
// FP32 AM contraction on the tensor cores (am_tc.cu): tiles of 128 x cells
// by `rows` (y, z) rows: 64-128 (two accumulator sets), 256 (one), or 0 =
// 128.  The halo columns x = 0 and
// gx + 1 are filled only where they are read: launch_am_halo_fill writes
// them into a temperature download buffer from the tables of the current
// step (they are computed every step when the layer flag lsindex is kept).
int launch_am_contract_tc(const KernelArgs &a, const AmParams &m, void *stream, int rows);
// the FP32 temperature as a tensor-store target (kernels.cu; map: a CUtensorMap)
bool encode_t32_store(void *map, const KernelArgs &a, int bx, int by);
int launch_am_halo_fill(const KernelArgs &a, const AmParams &m, double *dev_out, void *stream);
int am_tc_prepare();
long long am_ximg_size(int gx, int gy, int gz);  // floats of a.d.am_ximg
// Temperature of the next step for the AM model (tables + contraction);
// FP32 tables and sums in the FP32 form (`rows`: its contraction's tile).
int launch_temp_am(const KernelArgs &a, const AmParams &m, int precision, void *stream, Profiler *prof,
                   int rows = 0);
constexpr int RED_BLOCKS = 148 * 8;  // partial sums of k_reduce (red holds 2 per block + 1)
int launch_reduce(const KernelArgs &a, int precision, int what, double *host_out, void *stream, double *pinned);
// The TMA stencil launched with sumfs leaves each tile's sum of the new
// fraction solid in a.d.fs_part: stencil_parts is the tile count of the
// current launch (0 when the step runs another variant), stencil_parts_max
// the most any tile choice gives; launch_fold_fs folds them and copies the
// total to pinned memory (the caller synchronises).
long long stencil_parts(const KernelArgs &a, const TmaHolder &tma);
long long stencil_parts_max(const Geo &g);
int launch_fold_fs(const KernelArgs &a, long long nparts, void *stream, double *pinned);
// The same fold, written together with the control block (ctl) straight to
// pinned host memory through device-usable pointers; the caller
// synchronises, after which both are current on the host.
int launch_fold_fs_out(const KernelArgs &a, long long nparts, void *stream, double *host_sum, void *host_ctl);
int launch_fill_temperature(const KernelArgs &a, double *dev_out, void *stream);
int launch_compute_d(const KernelArgs &a, int precision, double *dev_out, void *stream);
int launch_repack(void *dst, long long dst_pitch, const void *src, long long src_pitch, int row_bytes, long long rows,
                  void *stream);
int launch_mask_captured(const KernelArgs &a, void *dev, int is_double, void *stream);
int launch_convert(const KernelArgs &a, int precision, int field, int to_device, double *dev_f64,
                   void *stream);
// the same between the field and FP64 values in the reference layout
int launch_convert_ref(const KernelArgs &a, int precision, int field, int to_device, double *ref_f64, void *stream);

// Frozen-CA replay and adjoint (adjoint.cu).  x0/x1: (ce, cl, fs) of one
// state; ts: the timestep of the step being replayed or differentiated.
constexpr int ADJ_SLOTS = 6;  // gradient slots: rl, D_xt, km, km_inv, k_inv, gibbs
int adj_nblocks(const Geo &g);
int launch_replay(const Geo &g, const Phys &p, int precision, const void *const x0[3], void *const x1[3],
                  const unsigned char *flags, const double *curv, unsigned long long ts, void *stream);
int launch_adj_step(const Geo &g, const Phys &p, int precision, const void *const x0[3], const void *ce1,
                    const unsigned char *flags, const double *curv, void *lce, const void *lcl1, const void *lfs1,
                    void *lcl0, void *lfs0, void *nu, double *partial, double *grad, unsigned long long ts,
                    void *stream);
int launch_adj_terminal(const Geo &g, int precision, double cinit_off, const void *ce, const double *target,
                        void *lce, void *lcl, void *lfs, double *partial, double *loss_out, void *stream);

}  // namespace mms

// the deck parameters a context was created with (mms_api.cu)
const mms_params &ctx_params(const mms_ctx *ctx);
