/*
 * mms.h — C ABI of mumatscale_b200, a B200-native implementation of the
 * muMatScale cellular-automaton solidification step.
 *
 * The reference's hot path is a set of C functions over one subblock
 * (SB_struct *lsp) and the global configuration (BB_struct *bp), called in a
 * fixed order by doiteration() (calculate.c:193-352) from the time loop
 * (loop.c:186-271).  This header replaces that boundary: a caller (the C
 * host loop, a Python script, another language through its FFI) creates one
 * context per GPU from the parsed input deck, advances it by whole
 * timesteps, and reads fields, reductions and the grain table back.  All
 * device memory belongs to the context; all host buffers belong to the
 * caller.  Calls on one context are ordered on one internal CUDA stream and
 * are not thread-safe for that context.  Every call returns an mms_status;
 * nothing in the library exits the process (the reference aborts through
 * error(), debug.h:54-58).
 *
 * The domain is the reference's global grid: NSubblocks x NCellsPerSB cells
 * held as one device-resident array with a one-cell halo, indexed exactly
 * like growth.c:70 on a single subblock:
 *     idx = k*(gdimy+2)*(gdimx+2) + j*(gdimx+2) + i,  i,j,k in [0, gdim+1]
 * with interior cells at 1..gdim.  When NSubblocks is not 1 1 1 the library
 * still runs one domain, and reproduces the per-rank orderings of the
 * reference's MPI run (grain ids, rand() streams, interface-list slots), so
 * results match the reference run on that many ranks.
 */
#ifndef MMS_H
#define MMS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MMS_ABI_VERSION 1

typedef enum mms_status {
    MMS_OK = 0,
    MMS_ERR_ARG = 1,             /* invalid argument or unsupported option */
    MMS_ERR_CUDA = 2,            /* a CUDA runtime call failed */
    MMS_ERR_NO_DEVICE = 3,       /* no usable sm_100 device */
    MMS_ERR_COURANT = 4,         /* Dsol/Dliq*dt/dx^2 > CourantLimit (growth.c:43-50) */
    MMS_ERR_NEGATIVE_CE = 5,     /* ce < 0 after diffusion (growth.c:163-165) */
    MMS_ERR_GRAIN_OVERFLOW = 6,  /* grain id beyond MaxTotGrains (grain.c:363-366) */
    MMS_ERR_DECK = 7,            /* input deck could not be parsed (read_ctrl.c) */
    MMS_ERR_IO = 8,              /* a file could not be written or read */
    MMS_ERR_TIMEOUT = 9,         /* a bounded device-side wait expired */
    MMS_ERR_STATE = 10,          /* call made in the wrong state */
    MMS_ERR_NOMEM = 11,          /* device or host allocation failed */
    MMS_ERR_SCRATCH_LIMIT = 12,  /* grid larger than the fixed device scratch of
                                    mms_reduce_field_noalloc (2^30 interior cells) */
    MMS_ERR_BOUNDS = 13,         /* a kernel index outside its buffer (only the
                                    bounds-checked build, libmms_b200_bounds.so,
                                    checks; the access is skipped) */
    MMS_ERR_SLAB_CAPACITY = 14   /* a slab's fixed per-step candidate row buffer
                                    (sized at creation from the sites it holds)
                                    was too small */
} mms_status;

typedef enum mms_precision {
    MMS_PREC_F64 = 0,  /* plain form: all fields FP64, bit-exact to the reference */
    MMS_PREC_F32 = 1   /* FP32 bulk ce/cl/fs; FP64 octahedra, thresholds, reductions */
} mms_precision;

/* FixedNuc x y z ax ay az threshold (read_ctrl.c:298-310); angles in degrees */
typedef struct mms_fixed_nuc {
    double x, y, z, ax, ay, az, threshold;
} mms_fixed_nuc;

/* NucVolume density[%] minx miny minz maxx maxy maxz threshold
 * (read_ctrl.c:311-330); density is stored as a fraction (value/100) */
typedef struct mms_nuc_volume {
    double density, minx, miny, minz, maxx, maxy, maxz, threshold;
} mms_nuc_volume;

/* The subset of BB_struct (globals.h:273-403) that the hot path, its setup
 * and the time loop read.  Names follow the reference. */
typedef struct mms_params {
    /* grid */
    int gnsbx, gnsby, gnsbz;          /* NSubblocks */
    int gsdimx, gsdimy, gsdimz;       /* NCellsPerSB */
    int padBndyX, padBndyY, padBndyZ; /* FaceCtrl: 1 = pad (mold), 0 = wrap */
    double origin_offset[3];
    double cellSize;
    double courant_limit;
    unsigned int base_random_seed;    /* RandSeedVal */
    /* time and termination */
    double ts_delt;                   /* TimeStep */
    double finish_time;               /* FinishTime (0 = off) */
    double fs_finish;                 /* FsFinish */
    /* growth */
    double fsgrow, rev_fsgrow;        /* FSGrow, 1/FSGrow */
    /* curvature */
    int tip_curv;                     /* TipCurvature */
    double gibbs_coef;                /* GibbsThomsonCoef */
    /* alloy */
    double liquidusTemp, solidusTemp, Cinit;
    double m_solute0, m_solute0_a, m_solute0_b, m_solute0_c;
    double part_coef, part_coef_a, part_coef_b, part_coef_c;
    double Dsol, Dliq;
    /* internal temperature (internal_temp_ctrl_t, globals.h:256-269) */
    double initialTemperature, gradient, velocity, grad_coef, velo_coef, cool_rate;
    /* laser analytical thermal model */
    int thermal_ana, am, amlayer, amtracks;
    double lpow, lv, lsd, lab, lhs, liniT, lthcon, lcp, rho, x0, y0, z0;
    /* nucleation */
    double maxGrainDensity, gnGaussCenter, gnGaussSigma;
    double maxGrainDensitySurf, gnGaussCenterSurf, gnGaussSigmaSurf;
    int doSurfaceNuc;                 /* MouldNuc */
    int gnUseOrientation;             /* GNOriented */
    uint64_t maxTotalGrains;          /* MaxTotGrains */
    /* output and time loop */
    int screenpfreq, data_write_freq, data_write_start, randomize_grains;
    int vis_format;                   /* 0 none, 1 VTK, 2 XDMF */
    char basefilename[256];
    /* nucleation lists from the deck (owned by whoever filled them) */
    const mms_fixed_nuc *fixed_nucs;
    int n_fixed_nucs;
    const mms_nuc_volume *nuc_volumes;
    int n_nuc_volumes;
    /* build options of this library */
    int precision;                    /* mms_precision */
    int device;                       /* CUDA device ordinal */
    /* No counterpart in the reference.  0: the volume and surface sites of
     * init_sb_nucleation (grain.c:930-1010) drawn on the host from each
     * rank's rand() stream, exactly as the reference draws them (O(cells)
     * host work).  1: drawn on the device from a counter-based generator
     * (Philox4x32-10) keyed by RandSeedVal: the same site densities
     * and threshold distributions, not the reference's sequence.  FixedNuc
     * and NucVolume sites are the reference's in both. */
    int site_setup;
    /* bp->checkpointfreq, which the reference's deck parser sets from
     * DataWriteStart (read_ctrl.c:594-600; it has no keyword of its own):
     * mms_run writes a checkpoint (mms_checkpoint_save to cp_main.mms in the
     * working directory, the counterpart of the reference's cp_main.h5) every
     * checkpoint_freq steps, as loop.c:244-247 calls writeCheckpoint;
     * 0 = never */
    int checkpoint_freq;
    /* No counterpart in the reference.  0: sb_curvature as the reference
     * writes it (curvature.c:81-405), quirks included: the normal is
     * normalised only when its length is 0 (curvature.c:194), a height
     * direction is chosen only when some normal component is exactly 0
     * (curvature.c:203), so curvature is 0 on generic interfaces, and the
     * upper smoothed face takes fs[idl] for fs[idu] (curvature.c:176).
     * 1: those three corrected (normalised when non-zero, the dominant
     * component always chosen, fs[idu]); for studies of the Gibbs-Thomson
     * term, not for parity. */
    int curvature_corrected;
} mms_params;

typedef enum mms_field {
    MMS_FIELD_CE = 0,            /* f64 [N]   equivalent concentration */
    MMS_FIELD_CL = 1,            /* f64 [N]   liquid concentration */
    MMS_FIELD_FS = 2,            /* f64 [N]   fraction solid */
    MMS_FIELD_GR = 3,            /* i32 [N]   grain id, 0 = liquid */
    MMS_FIELD_DC = 4,            /* f64 [3N]  octahedron centre offset, x,y,z per cell */
    MMS_FIELD_D = 5,             /* f64 [N]   half diagonal grow_octahedra gave cells that were
                                                solid at the last growth step, 0 elsewhere
                                                (download only) */
    MMS_FIELD_NUC_THRESHOLD = 6, /* f32 [N]   nucleation undercooling, +inf = no site */
    MMS_FIELD_TEMPERATURE = 7,   /* f64 [N]   temperature at the current timestep (download only) */
    MMS_FIELD_MOLD = 8,          /* i8  [N]   mold flag (download only) */
    MMS_FIELD_OGR = 9,           /* i32 [N]   grain ids before the last capture, the
                                                reference's ogr (growth.c:635-638; download only) */
    MMS_FIELD_CURV = 10          /* f64 [N]   curvature the last step used (TipCurvature 1;
                                                zeros otherwise; download only) */
} mms_field;

typedef enum mms_reduction {
    MMS_REDUCE_FS_FRACTION = 0,  /* computeFS (loop.c:173-183): sum min(1,fs) dx^3 / total volume */
    MMS_REDUCE_SOLID_VOLUME = 1, /* solid_volume (growth.c:971-978) */
    MMS_REDUCE_CE_SUM = 2        /* sum of ce over interior cells, compensated in FP64 */
} mms_reduction;

/* grain_t (globals.h:244-254) */
typedef struct mms_grain {
    double nuc_x, nuc_y, nuc_z;
    uint64_t nuc_timestep;
    double nuc_threshold;
    double rotmat[3][3];
    double rotang[3];
} mms_grain;

typedef struct mms_grain_summary {
    int num_grains;              /* bp->num_grains - 1 */
    double min_mm3, max_mm3, avg_mm3;
} mms_grain_summary;

typedef struct mms_ctx mms_ctx;

/* ---- configuration (read_ctrl.c) ------------------------------------------ */

/* set_defaults (read_ctrl.c:29-108). */
mms_status mms_params_default(mms_params *p);

/* read_config (read_ctrl.c:234-812) on top of *p, including GeoFileName /
 * MatFileName / AlloyPropsFile0 includes.  FixedNuc and NucVolume lines are
 * appended to heap arrays released by mms_params_free_lists(). */
mms_status mms_deck_read(const char *path, mms_params *p);
void mms_params_free_lists(mms_params *p);
/* sizeof(mms_params), for FFI bindings to check their layout */
size_t mms_params_size(void);

/* The reference's nucleation thresholds after setup (init_nucleation_sites,
 * grain.c:602-713, and init_sb_nucleation, grain.c:930-1010, every emulated
 * rank on its own rand() stream), written to thr_out[N] in the halo'd layout
 * (+inf where there is no site).  Host only: needs no CUDA device. */
mms_status mms_predraw_sites(const mms_params *p, float *thr_out);

/* ---- context lifetime ------------------------------------------------------ */

/* Allocates the device-resident domain and applies the reference's initial
 * state: allocateFields + SetupInitialConditions (setup.c:41-236), the
 * nucleation sites of init_nucleation_sites (grain.c:602-713) and
 * init_sb_nucleation (grain.c:930-1010), each emulated rank drawing from its
 * own srand(rank+1+seed) stream (ca_main.c:215).  Checks the Courant limit
 * (growth.c:43-50).  The step counter starts at 0 (findStartTime,
 * functions.c:512-576, always yields 0). */
mms_status mms_create(const mms_params *p, mms_ctx **out);
mms_status mms_destroy(mms_ctx *ctx);

/* ---- stepping (doiteration, calculate.c:193-352) --------------------------- */

/* Advances nsteps timesteps.  Each step increments the step counter and then
 * runs, in the reference's order: temperature, nucleation scan
 * (grain.c:1043), grain activation (grain.c:841), diffusion (growth.c:30),
 * Gibbs-Thomson curvature when TipCurvature is 1 (curvature.c:31),
 * fraction-solid change (growth.c:177), octahedron growth (growth.c:339),
 * interface list (growth.c:461) and capture (growth.c:574). */
mms_status mms_step(mms_ctx *ctx, int nsteps);

mms_status mms_get_timestep(mms_ctx *ctx, uint64_t *timestep);
/* bp->num_grains: grains created so far plus the "zero" grain */
mms_status mms_get_num_grains(mms_ctx *ctx, int *num_grains);

/* ---- fields and reductions ------------------------------------------------- */

/* Copies a whole halo'd field between the device and a caller buffer in the
 * layout described above.  N = (gdimx+2)(gdimy+2)(gdimz+2). */
size_t mms_num_cells(const mms_ctx *ctx);
mms_status mms_download(mms_ctx *ctx, mms_field field, void *host);
mms_status mms_upload(mms_ctx *ctx, mms_field field, const void *host);
/* computeFS / solid_volume (loop.c:173-183, growth.c:541-566) and the ce
 * sum, by a pass over the field (FP64, compensated). */
mms_status mms_reduce(mms_ctx *ctx, mms_reduction what, double *out);

/* mms_step followed by mms_reduce, with one synchronisation: the reference
 * loop's doiteration followed by computeFS at a screen-output step
 * (loop.c:227-234).  For the fraction-solid reductions the last step's
 * stencil also leaves one sum per tile, and those few thousand values are
 * folded instead of reading the field again (mms_reduce does the same until
 * the next call that steps or writes fields).  Both are FP64 sums within a
 * few ulps of each other, in different orders. */
mms_status mms_step_reduce(mms_ctx *ctx, int nsteps, mms_reduction what, double *out);

/* Allocation-free form of mms_reduce over a caller-owned field.  It has no
 * counterpart in the reference (whose reductions run on host arrays); it is
 * for callers that may not allocate device memory where they reduce.
 *   field       device pointer: ce or fs of a (gdimx, gdimy, gdimz) grid in
 *               the halo'd layout above, FP64 (dtype MMS_PREC_F64) or FP32
 *               (MMS_PREC_F32) elements, absolute values as mms_download
 *               returns them
 *   out         device pointer to one double, written asynchronously on
 *               cuda_stream (a cudaStream_t; NULL = the legacy default stream)
 * The result is the same sum as mms_reduce's, compensated in FP64, in a
 * different summation order.  Intermediates live in a fixed 1 MiB device
 * array of the library: grids above 2^30 interior cells return
 * MMS_ERR_SCRATCH_LIMIT.  The array is shared by all calls on a device, so
 * calls that may overlap on one device (unordered streams, several host
 * threads) race.  The array's address is looked up on the first call in
 * each CUDA context (and again when a call finds another context current on
 * that device, e.g. after a reset): that first call should come before any
 * stream capture in the context.  Kernels are launched with
 * cudaLaunchKernel and its return code checked, so a pending error of the
 * caller's own CUDA work is not cleared.  Nothing is allocated. */
mms_status mms_reduce_field_noalloc(const void *field, mms_precision dtype,
                                    int gdimx, int gdimy, int gdimz,
                                    mms_reduction what, double cell_size,
                                    double *out, void *cuda_stream);

/* ---- sites and orientations ------------------------------------------------ */

/* Replaces every nucleation threshold: cells listed get the given threshold
 * (0-based global interior cell coordinates), every other cell +inf.  This is
 * what a pre-drawn site list injects in place of init_sb_nucleation. */
mms_status mms_set_sites(mms_ctx *ctx, int64_t n, const int32_t *gxyz,
                         const float *thresholds);
/* Orientation override for grains that nucleate at the listed cells: their
 * rotation matrix (row-major 3x3) replaces the one createGrains would build
 * (grain.c:348-425); rand() is still consumed as in the reference. */
mms_status mms_set_site_orientations(mms_ctx *ctx, int64_t n, const int32_t *gxyz,
                                     const double *rotmat9);

/* Failure-detection test hook, no counterpart in the reference (whose
 * failures abort the process, debug.h:54-58).  From the next step on, the
 * interface-list block at list position `block` publishes no status word, so
 * the decoupled look-back of the block after it waits for a word that nothing
 * writes; that wait gives up after `polls` polls (0: 2^22, about a second)
 * and the step returns MMS_ERR_TIMEOUT, with no device fault and the device
 * usable.  block = -1 turns the hook off.  The context is in error after such
 * a step; destroy it. */
mms_status mms_test_hold_list_block(mms_ctx *ctx, int block, unsigned polls);

/* A pre-filled microstructure (for example a substrate of columnar grains):
 * defines grains 1..n with the given row-major rotation matrices, so that
 * nucleated grains continue from id n+1.  Only before the first step; the
 * caller then uploads gr (ids 1..n), fs and the concentrations of the
 * cells those grains fill.  Their grain records carry no nucleus. */
mms_status mms_set_grains(mms_ctx *ctx, int n, const double *rotmat9);

/* ---- grain table and results ----------------------------------------------- */

mms_status mms_get_grains(mms_ctx *ctx, int first, int count, mms_grain *out);
/* output_grains (grain.c:751-833): writes <basefilename>_grains.csv when path
 * is non-NULL and returns the summary line's numbers. */
mms_status mms_output_grains(mms_ctx *ctx, const char *path, mms_grain_summary *out);

/* ParaView output in the layout of io_vtk.c: <base>_<ts>.pvtu naming one
 * piece per subblock, <base>_<sbid>/<ts>.vtu with the cell arrays
 * Temperature (Float64) and Grain (Int32) on hexahedral cells
 * (writepvtu/writevtu, io_vtk.c:39-463), plain-text encoding.  base NULL =
 * the deck's BaseFileName. */
mms_status mms_write_vtk(mms_ctx *ctx, const char *base);
/* The same files from caller arrays in the halo'd layout (host only). */
mms_status mms_write_vtk_arrays(const mms_params *p, const char *base, int64_t timestep,
                                const double *temperature, const int32_t *gr);
/* XDMF output as xdmf_writeMain + xdmf_writeSubblocks (io_xdmf.c:141-673):
 * <base>_ts.xmf, the time series of every write since the first one to this
 * base; <base>_r<rank>/<ts>.raw per emulated rank (Temperature, CE as
 * float32, Grain as int32, FracSolid as float32, each the subblock's interior
 * with z slowest, in that order); <base>_gbl.raw (with RandomizeGrains the
 * grain renumbering as uint64, then the grain angles X, Y, Z as float32).
 * The reference writes these datasets with HDF5, which is absent here: the
 * index addresses the raw files with Format="Binary" and Seek offsets.
 * With RandomizeGrains, a write after the grain count grew draws a new
 * renumbering from rank 0's rand() stream (getRenumberArray,
 * io_xdmf.c:344-375), which shifts rank 0's later orientation draws exactly
 * as in the reference.  base NULL: the deck's BaseFileName.  mms_run writes
 * these (or VTK) itself for DataFormat XDMF (VTK) with DataWriteFreq > 0.
 * Not on a slab of a split domain. */
mms_status mms_write_xdmf(mms_ctx *ctx, const char *base);
/* The files of one write from halo'd host arrays (reference layout): series
 * lists the timesteps of the time series, the last being this write's;
 * rotang [num_grains][3]; renumber NULL unless RandomizeGrains. */
mms_status mms_write_xdmf_arrays(const mms_params *p, const char *base, const int64_t *series, int nseries,
                                 const double *temperature, const double *ce, const int32_t *gr, const double *fs,
                                 int num_grains, const double *rotang, const uint64_t *renumber);
/* The grain renumbering of the last XDMF write (count entries; up to
 * capacity copied to out). */
mms_status mms_xdmf_renumbering(mms_ctx *ctx, int capacity, uint64_t *out, int *count);

/* Raw checkpoint of a context (device layout, this library's format): every
 * array a later step reads, the grain table, the orientation tables and the
 * state of the per-rank random streams, the sites and orientation
 * overrides.  Loading into a context created from the same deck and form
 * continues exactly as the saved context would have (the role of
 * checkpoint.c's restart, checkpoint.c:955-1244, without HDF5). */
mms_status mms_checkpoint_save(mms_ctx *ctx, const char *path);
/* the file mms_run writes every checkpoint_freq steps, and mmsb200 -r reads */
#define MMS_CHECKPOINT_FILE "cp_main.mms"
mms_status mms_checkpoint_load(mms_ctx *ctx, const char *path);

/* ---- the time loop (loop.c:186-271) ----------------------------------------- */

/* Runs the reference time loop to its termination (FinishTime / FsFinish,
 * checked with the fraction solid refreshed every ScreenPFreq steps),
 * printing the reference's screen lines and grain summary to stdout when
 * verbose is non-zero. */
mms_status mms_run(mms_ctx *ctx, int verbose);

/* ---- streams and timing ----------------------------------------------------- */

/* Runs all of this context's work on the caller's CUDA stream (a
 * cudaStream_t passed as a plain pointer; NULL restores the context's own
 * stream).  The stream must outlive its use by the context. */
mms_status mms_set_stream(mms_ctx *ctx, void *cuda_stream);
/* When on, every kernel launch is bracketed by CUDA events on the launching
 * stream, and per-kernel device time accumulates for mms_kernel_stats. */
mms_status mms_set_profiling(mms_ctx *ctx, int on);
/* Kernel ids 0..mms_kernel_count()-1; name and accumulated statistics. */
int mms_kernel_count(void);
const char *mms_kernel_name(int id);
mms_status mms_kernel_stats(mms_ctx *ctx, int id, double *total_ms, uint64_t *launches);

/* Tile of the diffusion + fs-change stencil: cells per thread along x (1 or
 * 2: CTA tiles of 32 x 8 or 64 x 8 cells) and planes per CTA along z (1-64;
 * 0 = chosen from the grid size).  Results do not depend on the tile. */
mms_status mms_set_stencil_tile(mms_ctx *ctx, int cells_per_thread, int zchunk);
mms_status mms_get_stencil_tile(const mms_ctx *ctx, int *cells_per_thread, int *zchunk);
/* FP32 form, moving-source (AM) temperature: rows per tile of its
 * tensor-core contraction (tiles of 128 x cells by `rows` (y, z) rows): 64 to
 * 128 in steps of 16, 256, or 0 (the default) = 256 when the grid holds at
 * least two 256-row tiles per SM, else 128.  Results do not depend on it. */
mms_status mms_set_am_tile(mms_ctx *ctx, int rows);
mms_status mms_get_am_tile(const mms_ctx *ctx, int *rows);
/* Times every tile candidate on shadow copies of the fields the stencil
 * writes (the domain's state is left as it was), keeps the fastest by median
 * of `reps` launches and returns it (any output pointer may be NULL).  For
 * the FP32 form of the moving-source (AM) temperature model it also picks
 * the tensor-core contraction's tile (128 x cells by 128 or 256 rows), timed
 * on a shadow of the temperature field.  Results do not depend on either
 * choice. */
mms_status mms_autotune(mms_ctx *ctx, int reps, int *cells_per_thread, int *zchunk, double *best_ms);

/* ---- batched independent domains --------------------------------------------- */

/* No counterpart in the reference.  n independent domains (each its own
 * deck: sizes, cooling, nucleation) stepped together on one device: per
 * step one CUDA graph with every domain's nucleation, activation, list and
 * capture as parallel branches and one persistent stencil launch over the
 * tiles of all domains.  All params[i] must share precision and device.
 * Each domain's state is exactly what mms_step would give it alone. */
typedef struct mms_batch mms_batch;
mms_status mms_batch_create(int n, const mms_params *params, mms_batch **out);
mms_status mms_batch_destroy(mms_batch *b);
int mms_batch_size(const mms_batch *b);
/* The i-th domain's context, for uploads, downloads, reductions and grain
 * records (not for mms_step while it belongs to the batch). */
mms_ctx *mms_batch_domain(mms_batch *b, int i);
mms_status mms_batch_step(mms_batch *b, int nsteps);
/* Stencil tile of the persistent launch (as mms_set_stencil_tile). */
mms_status mms_batch_set_stencil_tile(mms_batch *b, int cells_per_thread, int zchunk);
mms_status mms_batch_get_stencil_tile(const mms_batch *b, int *cells_per_thread, int *zchunk, int *grid);
/* Times the persistent stencil for every tile candidate on shadows of the
 * fields it writes and keeps the fastest. */
mms_status mms_batch_autotune(mms_batch *b, int reps, int *cells_per_thread, int *zchunk, double *best_ms);
uint64_t mms_batch_kernel_launches(const mms_batch *b);
const char *mms_batch_last_error(const mms_batch *b);

/* ---- one domain split into z-slabs over devices ------------------------------- */

/* The reference runs one domain as NSubblocks MPI ranks that exchange halo
 * planes and grain lists inside doiteration (calculate.c:193-352; ranks
 * numbered x fastest, functions.c:310,327).  Here the domain is cut
 * into nslabs z-slabs of whole subblock layers (nslabs <= NSubblocks z),
 * one context per slab, each on its own device or all on one: slab s owns
 * layers [s nz / nslabs, (s + 1) nz / nslabs) and their emulated ranks, so
 * their random streams, interface lists and dc_tmp slots never cross a
 * slab.  Stepped together, the slabs give the single context's fields,
 * grain ids and grain records bit for bit.  Each slab's fields, downloads
 * and reductions are its own (reference layout of the slab: nz = its
 * layers); coordinates in mms_set_sites and mms_set_site_orientations are
 * the whole domain's.  Not with TipCurvature (its stencil reaches three
 * planes) nor with a periodic z axis; no adjoint on a slab. */
typedef struct mms_slab_layout {
    int nslabs, slab;
    int z_begin;     /* first interior z cell of the slab in the whole domain (0-based) */
    int z_cells;     /* interior z cells */
    int rank_begin;  /* first emulated rank (x fastest, then y, then z) */
    int rank_count;
} mms_slab_layout;

/* The layout alone, from the whole domain's parameters (no device). */
mms_status mms_slab_layout_of(const mms_params *global, int nslabs, int slab, mms_slab_layout *out);
/* Context of slab `slab` of the domain `global` describes (its device:
 * global->device). */
mms_status mms_slab_create(const mms_params *global, int nslabs, int slab, mms_ctx **out);
mms_status mms_slab_get_layout(const mms_ctx *ctx, mms_slab_layout *out);
/* Steps all slabs of a domain in this process: slabs[s] is slab s.  The
 * exchanges are device copies (peer copies between devices) ordered by
 * events on the slabs' streams. */
mms_status mms_slab_group_step(mms_ctx *const *slabs, int nslabs, int nsteps);

/* One process per device: the caller runs the exchanges (e.g. with NCCL).
 * A step that starts at timestep t is
 *   mms_slab_launch(ctx, 0, 0); exchange point 0;
 *   mms_slab_launch(ctx, 1, 0); exchange point 1;
 *   mms_slab_launch(ctx, 2, 0);
 * with the transfers mms_slab_exchange_plan lists for (point, t), issued on
 * the context's stream (mms_set_stream).  Halo entries: send `bytes` from
 * `send` to slab `peer` and receive as many from it into `recv`; a slab's
 * entries for peer q and q's entries for it pair up in list order.  Gather
 * entry: every slab contributes `bytes` from `send`; `recv` receives the
 * nslabs contributions in slab order.  After some steps, mms_slab_poll
 * reports whether activation stalled for want of pre-drawn orientations;
 * every slab then stalls at the same step, and the steps launched after it
 * did nothing.  mms_slab_refill on every slab, then the stalled step again
 * with mms_slab_launch(ctx, 0, 1) in place of phase 0, resumes. */
typedef enum mms_xfer_kind { MMS_XFER_HALO = 0, MMS_XFER_GATHER = 1 } mms_xfer_kind;
typedef struct mms_slab_xfer {
    int kind;        /* mms_xfer_kind */
    int peer;        /* halo: the neighbouring slab; gather: -1 */
    void *send;      /* device memory of this context */
    void *recv;
    uint64_t bytes;
} mms_slab_xfer;
mms_status mms_slab_launch(mms_ctx *ctx, int phase, int resume);
mms_status mms_slab_exchange_plan(mms_ctx *ctx, int point, uint64_t timestep, mms_slab_xfer *out, int max,
                                  int *n);
mms_status mms_slab_poll(mms_ctx *ctx, uint64_t *timestep, int *stalled);
/* One process per device over NCCL (the role of the reference's MPI
 * exchanges inside doiteration, calculate.c:232-337, and of the grain
 * Allgatherv, grain.c:892-904).  The library does not link NCCL: it loads
 * the entry points from nccl_path (NULL: "libnccl.so.2", which finds a copy
 * the process has already loaded, e.g. torch's).
 *   mms_slab_nccl_unique_id  one rank makes the 128-byte ncclUniqueId, which
 *                            the caller sends to every rank of the group
 *   mms_slab_nccl_init       every slab context (slab index = NCCL rank)
 *                            joins the communicator
 *   mms_slab_nccl_step       nsteps steps: the three launch phases, with the
 *                            two exchange points as NCCL groups (halo planes
 *                            as send/recv with the neighbouring slabs, the
 *                            candidate and new-grain lists as all-gathers),
 *                            all on the context's stream; every 64 steps an
 *                            all-reduce checks that every slab is at the same
 *                            step and stall state, and a shortage of
 *                            pre-drawn orientations is refilled and resumed
 *                            on every slab.  Every rank calls it with the
 *                            same nsteps.
 *   mms_slab_nccl_reduce     the whole domain's reduction: this slab's sum,
 *                            all-reduced over the group. */
mms_status mms_slab_nccl_unique_id(const char *nccl_path, void *id128);
mms_status mms_slab_nccl_init(mms_ctx *ctx, const char *nccl_path, const void *id128);
mms_status mms_slab_nccl_step(mms_ctx *ctx, int nsteps);
mms_status mms_slab_nccl_reduce(mms_ctx *ctx, mms_reduction what, double *out);
mms_status mms_slab_refill(mms_ctx *ctx);

/* ---- adjoint (frozen cellular automaton) -------------------------------------- */

/* No counterpart in the reference.  Gradients of L = 1/2 sum over interior
 * cells of (ce - target)^2 after a recorded run, with respect to D_l
 * (Dliq), k (part_coef) and the Gibbs-Thomson coefficient, through the
 * diffusion (growth.c:69-162) and fraction-solid change (growth.c:220-273)
 * of every step, with the cellular automaton frozen: each cell's
 * fs_change branch, nucleation, capture and the curvature are those of the
 * recorded run.  Analytic temperature models only (not AnalyticalThermal 1). */
typedef struct mms_adjoint_result {
    double loss;
    double dL_dDliq;
    double dL_dpart_coef;
    double dL_dgibbs;
    int64_t steps;        /* recorded steps differentiated through */
} mms_adjoint_result;

/* Runs nsteps ordinary steps while recording, per step, the branch every
 * cell took and (with TipCurvature) its curvature, and the state (ce, cl,
 * fs) every checkpoint_every steps, starting with the current one.  Replaces
 * an earlier record. */
mms_status mms_adjoint_record(mms_ctx *ctx, int nsteps, int checkpoint_every);
/* Loss and gradient for the recorded run; target_ce in the halo'd layout
 * (FP64).  Each segment between checkpoints is recomputed from its
 * checkpoint by frozen replay, then differentiated backwards. */
mms_status mms_adjoint_gradient(mms_ctx *ctx, const double *target_ce, mms_adjoint_result *out);
/* Loss of the frozen replay of the whole recorded run from its first
 * checkpoint with Dliq, part_coef and GibbsThomsonCoef multiplied by
 * scale[0..2] (scale 1,1,1 reproduces the recorded run): the function the
 * gradient differentiates, for finite-difference checks. */
mms_status mms_adjoint_replay_loss(mms_ctx *ctx, const double *target_ce, const double scale[3], double *loss);
/* Frees the record. */
mms_status mms_adjoint_release(mms_ctx *ctx);

/* ---- diagnostics ----------------------------------------------------------- */
const char *mms_status_string(mms_status s);
/* The most recent error message on this context (empty when none). */
const char *mms_last_error(const mms_ctx *ctx);
/* Number of device kernels this context has launched since creation. */
uint64_t mms_kernel_launches(const mms_ctx *ctx);
/* 1 when the stencil runs its TMA-fed variant (descriptors encoded), 0 when
 * it uses its plain-load variant. */
int mms_uses_tma(const mms_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* MMS_H */
