/*
 * bsgpu.h - C ABI of the B200 (sm_100a) single-particle reconstruction and
 * projection-matching library (libbsgpu.so).
 *
 * The reference (Bsoft) has no plugin or FFI layer; its boundary for this
 * path is the C++ library call surface that `breconstruct` / `brefine`
 * drive.  Each entry point below names the reference interface it replaces:
 *
 *   bsg_recon_create     <- per-map set-up in particle_reconstruct
 *                           (bsoft/src/mg/mg_reconstruct.cpp:100-125) and the
 *                           plan created in breconstruct.cpp:268
 *   bsg_recon_insert     <- particle_reconstruct's per-particle loop
 *                           (mg_reconstruct.cpp:143-229): pad, fft, origin
 *                           shift, img_ctf_apply_complex, fspace_pack_2D
 *                           (bsoft/include/mg_reconstruct.h:16-19,
 *                            bsoft/include/Bimage.h:934-939)
 *   bsg_recon_finish     <- img_reconstruction_sum_weigh (mg_reconstruct.h:20,
 *                           mg_reconstruct.cpp:266-361) + fft_back
 *                           (Bimage.h:903-908) + filter_sinc
 *                           (breconstruct.cpp:328-359)
 *   bsg_recon_add_partial <- the partial-map sum in img_reconstruction_sum_weigh
 *                           (mg_reconstruct.cpp:263-324), across GPUs
 *   bsg_recon_fsc        <- Bimage::fsc (bsoft/src/img/Bimage_resolution.cpp:330-406)
 *   bsg_particle_spectra <- the 2-D half of particle_reconstruct
 *                           (Bimage::fft + phase_shift_to_origin +
 *                            img_ctf_apply_complex), exposed on its own
 *
 * Conventions: every function returns 0 (BSG_OK) or a negative BSG_ERR_*
 * code and leaves a message for bsg_last_error() (thread-local), the way the
 * reference returns NULL / <0 after error_show (bsoft/src/util/utilities.cpp:745).
 * Host buffers are caller-owned; a context owns its device memory and its
 * CUDA streams (bsg_recon_stream returns the one the gridding and finishing
 * run on), and is used by one host thread at a time.
 */
#ifndef BSGPU_H
#define BSGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BSG_OK          0
#define BSG_ERR_ARG    -1   /* invalid argument / unsupported size          */
#define BSG_ERR_CUDA   -2   /* CUDA runtime error                           */
#define BSG_ERR_STATE  -3   /* call out of order / context unusable         */
#define BSG_ERR_NOMEM  -4   /* device or host allocation failed             */
#define BSG_ERR_NODEV  -5   /* no usable sm_100 device                      */

/* flags */
#define BSG_DEVICE_PTR  1   /* image / output pointers are device pointers  */
#define BSG_SINC        2   /* bsg_recon_finish: apply the trilinear sinc   */

/* Per-particle record: 32 doubles, host layout (see bsoft_b200/plan.py):
 *   [0..1]  origin x, y (pixels)              Bparticle::ori
 *   [2..3]  background circle centre (pixels) image origin from the file
 *   [4..12] rotation matrix, row-major        View::matrix (View.h:153-156)
 *   [13]    particle pixel size (angstrom)
 *   [14]    frequency scale = 1/magnification (1 if none)
 *   [15]    particle weight (1, or selection number when bootstrapping)
 *   [16..22] CTF: abw00 abw20 abw22 abw2m2 abw40 abw11 abw1m1 (ctf.h:321-351)
 *   [23]    half-map index (0 or 1)
 *   [24..25] image normalisation: every pixel becomes v * [24] + [25]
 *            (float) before the background and padding, as
 *            rescale_to_avg_std(0, 1) under breconstruct -rescale
 *            (mg_reconstruct.cpp:155); [24] = 0: none
 */
#define BSG_PARTICLE_DOUBLES 32

typedef struct {
    int    n;            /* particle box edge                                 */
    int    ft;           /* padded transform edge: power of two in [32, 1024] */
    int    map;          /* map edge N: even, 8 <= N <= 512, N <= ft          */
    double map_sampling; /* angstrom / voxel                                  */
    double hi_res;       /* resolution limit (angstrom) after check_resolution */
    int    interp;       /* 0 nearest, 1 weighted nearest, 2 trilinear        */
    int    ctf_action;   /* 0 none, 1 flip, 2 apply, >= 3 Wiener-type         */
    double wiener;       /* Wiener factor                                     */
    int    nmaps;        /* 1 full map, 2 two half maps, 3 full + half maps   */
    int    fom;          /* 1: accumulate power and weight^2 as well          */
    int    batch;        /* particles per device batch, 0 = automatic         */
    int    device;       /* CUDA device ordinal                               */
} bsg_recon_config;

typedef struct bsg_recon bsg_recon;

/* Kernel timing collected with CUDA events on the context's stream
 * (enabled with bsg_recon_set_timing). */
typedef struct {
    long   launches;          /* all kernels this library launched          */
    long   insert_launches;   /* gridding kernel launches                   */
    double insert_ms;         /* summed device time of the gridding kernel  */
    double fft2d_ms;          /* background + row + column passes, elapsed on
                                 their stream (they overlap the gridding)   */
    double h2d_ms;            /* host-to-device copies of particle images   */
    long   particles;         /* particles inserted                         */
} bsg_recon_stats;

int  bsg_recon_create(const bsg_recon_config* cfg, bsg_recon** out);
void bsg_recon_destroy(bsg_recon* r);

/* Insert nparts particles: images (nparts x n x n float32, x fastest) and
 * params (nparts x BSG_PARTICLE_DOUBLES, host).  Accumulation order is fixed
 * (particle order, then pixel order), so results are bitwise reproducible.
 * The call is asynchronous: the images (host, where pinned buffers are read
 * by an asynchronous copy, or device with BSG_DEVICE_PTR, which must be
 * complete when the call is made) stay unchanged until
 * bsg_recon_synchronize.  One batch's 2-D transforms overlap the previous
 * batch's gridding. */
int  bsg_recon_insert(bsg_recon* r, const float* images, const double* params,
                      long nparts, int flags);

/* Weigh map imap (0 full, 1/2 half maps; see nmaps), shift the origin to the
 * centre, inverse-transform and (with BSG_SINC) apply the sinc weighting.
 * map_out: N^3 float32 real-space map; fom_out (optional, needs fom = 1):
 * N^3 float32 signal-to-noise map (fspace_reconstruction_snr). */
int  bsg_recon_finish(bsg_recon* r, int imap, float* map_out, float* fom_out, int flags);

/* Accumulated sums of half h (0/1; 0 when nmaps == 1): complex volume
 * (2*N^3 doubles) and weights (N^3 doubles), reference index order (the
 * accumulators are kept in FP64 on the device; with half-space gridding,
 * see bsg_recon_set_half_space, the map's sums are formed on the way out).
 * With BSG_DEVICE_PTR and half-space gridding, give both outputs. */
int  bsg_recon_accumulators(bsg_recon* r, int half, double* vol_out, double* weight_out, int flags);

/* Add another reconstruction's partial sums into half h of this context:
 * the reference's partial-map sum before weighing (img_reconstruction_sum_
 * weigh, bsoft/src/mg/mg_reconstruct.cpp:263-324, over the per-thread maps
 * of breconstruct.cpp:268-305).  With particles split across GPUs, each
 * shard's accumulators (bsg_recon_accumulators) are added, in shard order,
 * into one context, which then finishes the map; the sum is FP64, so the
 * result depends only on that order.  vol: 2*N^3 doubles, weight: N^3;
 * power and weight2 (N^3 each, both or neither) need fom = 1.  Host or
 * device (BSG_DEVICE_PTR) pointers; returns when the sums have been added.
 * A context in half-space form (bsg_recon_set_half_space) first turns its
 * sums into the full map's. */
int  bsg_recon_add_partial(bsg_recon* r, int half, const double* vol, const double* weight,
                           const double* power, const double* weight2, int flags);

/* Fourier shell correlation of the two weighed half-map transforms
 * (nmaps >= 2) as Bimage::fsc(Bimage*) forms it: shells linearly
 * interpolated, sampling ratio 1, FSC[0] = 1, shells from
 * map * sampling / hi_res on are 0.  nshell doubles. */
int  bsg_recon_fsc(bsg_recon* r, int nshell, double* fsc_out);

/* Reconstruction statistics of map imap (0 full, 1/2 halves) as
 * img_reconstruction_sum_weigh reports them (bsoft/src/mg/mg_reconstruct.cpp:
 * 328-349) after fspace_reconstruction_weigh (bsoft/src/img/
 * Bimage_reconstruct.cpp:486-515): the Friedel symmetry residual
 * (Bimage::friedel_check, bsoft/src/img/Bimage_fspace.cpp:2024), the
 * coverage (voxels with weight > 1e-30) and its percentage of the sphere of
 * radius maxrad + 1, and the shell table of fspace_reconstruction_stats
 * (Bimage_reconstruct.cpp:526-599): rows for radii 1 .. maxrad - 1 with
 * maxrad = map * sampling / resolution (resolution: breconstruct's limit
 * before any check, the sampling by default), columns BSG_STATS_COLUMNS:
 * radius, s (1/A), resolution (A), weight, power, signal, noise, SNR, FSC;
 * and the SNR(0.5) and FSC(0.3) resolution estimates (A, 0 when not
 * crossed).  The radial averages follow Bimage::radial and
 * fspace_radial_power (linear interpolation between shells); where the
 * reference reads past the end of its arrays (radii >= map / 2 for the
 * channel averages, radii beyond the checked resolution for the power), the
 * values are 0, as it prints them.  Needs fom = 1 (the power and weight^2
 * channels); computed on the host from the FP64 sums.  table: max_rows x
 * BSG_STATS_COLUMNS doubles (rows beyond max_rows are dropped). */
#define BSG_STATS_COLUMNS 9
typedef struct {
    double friedel;          /* Friedel symmetry residual                      */
    long   coverage;         /* voxels with weight > 1e-30                     */
    double coverage_pct;     /* coverage / (4/3 pi (maxrad + 1)^3) x 100       */
    double res_snr;          /* SNR(0.5) resolution estimate (angstrom)        */
    double res_fsc;          /* FSC(0.3) resolution estimate (angstrom)        */
    int    rows;             /* shell rows (maxrad - 1)                        */
} bsg_recon_shell_stats;
int  bsg_recon_statistics(bsg_recon* r, int imap, double resolution, bsg_recon_shell_stats* out, double* table,
                          int max_rows);

/* The 2-D stage alone: padded FFT, origin shift and CTF of nparts images;
 * out = nparts x ft x ft complex64 (interleaved), reference pixel order. */
int  bsg_particle_spectra(bsg_recon* r, const float* images, const double* params,
                          long nparts, float* out, int flags);

/* Gridding tile shape (0: 8x8x8 (default), 1: 16x16x4, 2: 16x8x8,
 * 3: 16x16x8 without FOM).  bsg_recon_autotune times every shape on the
 * given particles, keeps the fastest and then clears the accumulators: call
 * it before inserting.  ms_out (optional) receives one time per shape
 * (-1 where the shape does not apply); best_out the chosen shape.  The
 * reference has no counterpart (it has no tunable tiling). */
int  bsg_recon_set_tile_shape(bsg_recon* r, int shape);

/* Half-space gridding (on by default; applies to trilinear insertion
 * without the FOM channels).  A real particle image has a Hermitian
 * transform, so the sums P of the pixels whose Friedel mate is in the
 * stored transform satisfy P(-v) = conj(P(v)), P_w(-v) = P_w(v); the
 * unpaired pixels (row and column -ft/2) make sums U of their own.  The
 * tiles below zsplit (the first multiple of 8 above N/2) grid P and,
 * apart, U; the tiles at or above it grid only U; every read of the sums
 * (finish, FSC, bsg_recon_accumulators) gives P(v) + U(v) below the split
 * and conj(P(-v)) + U(v) above it: the full map's contributions, none
 * subtracted, for about half the gridding work.  The reference grids the
 * full map (fspace_pack_2D, bsoft/src/img/Bimage_reconstruct.cpp:112-174).
 * enable 0 turns the accumulators into the full map's sums and grids the
 * full map from then on; switching on needs empty accumulators (before
 * inserting or after bsg_recon_reset).  bsg_recon_add_partial and a batch
 * with Ewald surfaces (not Hermitian) switch it off the same way.
 * zsplit_out (optional): the split in use, 0 for the full map. */
int  bsg_recon_set_half_space(bsg_recon* r, int enable, int* zsplit_out);

/* Point-group symmetry during reconstruction (breconstruct -symmetry, mode
 * 0): Bimage::fspace_pack_2D(p, View, sym, ...) (bsoft/src/img/
 * Bimage_reconstruct.cpp:248-266) inserts each particle once per view of
 * symmetry_get_all_views (bsoft/src/util/symmetry.cpp:277-319); the view
 * made by the group element q from the particle's view v has the matrix
 * M(q) M(v).  ops: nops rotation matrices M(q) (row-major, the identity
 * first, in the reference's generation order); every later insert grids
 * each particle with matrix M(q) R for every operator, all copies from the
 * particle's one transform.  nops <= 1 restores C1. */
int  bsg_recon_set_symmetry(bsg_recon* r, const double* ops, int nops);

/* Point-group symmetry after reconstruction (breconstruct -symmetry with
 * -mode 1): the particles are inserted once (C1), and bsg_recon_finish
 * applies Bimage::symmetrize(sym, 1) (bsoft/src/img/Bimage_symmetry.cpp:
 * 31-100, bsoft/src/breconstruct.cpp:335) to the real-space map before the
 * sinc weight: for each generating operation, in order, the map becomes the
 * sum of itself and its order - 1 rotations about the axis through the map
 * centre (trilinear resampling as Bimage::interpolate does it, the map's
 * background outside), then every value is divided by the group order.
 * axes: nops axes (3 doubles each, as Bsymmetry defines them, e.g. 1,1,1
 * for the 3-fold of T; normalised here as the reference normalises them),
 * orders: nops orders 1..9, nops <= 8; nops = 0 turns it off. */
int  bsg_recon_set_symmetrize(bsg_recon* r, const double* axes, const int* orders, int nops);

/* breconstruct -rescale avg,std: bsg_recon_finish rescales the real-space
 * map (after the inverse transform and any symmetrization, before the sinc
 * weight) to the given average and standard deviation from its own
 * (Bimage::rescale_to_avg_std, bsoft/src/img/Bimage_rescale.cpp:163-182;
 * bsoft/src/breconstruct.cpp:336).  std <= 0 turns it off. */
int  bsg_recon_set_rescale(bsg_recon* r, double avg, double std);
int  bsg_recon_autotune(bsg_recon* r, const float* images, const double* params, long nparts,
                        int flags, double* ms_out, int* best_out);

int  bsg_recon_set_timing(bsg_recon* r, int enable);
int  bsg_recon_get_stats(bsg_recon* r, bsg_recon_stats* st);
int  bsg_recon_reset(bsg_recon* r);          /* zero the accumulators        */
int  bsg_recon_synchronize(bsg_recon* r);
void* bsg_recon_stream(bsg_recon* r);        /* the context's cudaStream_t  */

/* The 2-D stage without any device allocation by the library, for callers
 * that manage all device memory themselves (a pipeline that reserves its
 * memory up front, or a host that forbids device allocations after start-up).
 * No counterpart in the reference: it never runs on a GPU.
 *
 * d_images (nparts x n x n float32) and d_out (nparts x ft x ft complex64,
 * the same order as bsg_particle_spectra) are device pointers owned by the
 * caller; params is the host record array, converted and sent to the
 * device in one copy from ordinary host memory (CUDA orders that copy with
 * `stream` and stages it before the call returns).  Work goes to `stream` (a
 * cudaStream_t, NULL for the default stream).  The intermediate data use a
 * fixed scratch area of BSG_NOALLOC_SCRATCH_BYTES inside the library, held
 * on every GPU that loads it until exit; a call needing more (too many or
 * too large particles) fails with BSG_ERR_ARG and says how many fit.  The
 * first call on a device looks up that area's address: make it before any
 * stream capture.  Calls share the area, so calls whose work overlaps on
 * the GPU race: serialise them. */
#define BSG_NOALLOC_SCRATCH_BYTES ((size_t)64 << 20)
int  bsg_particle_spectra_noalloc(const bsg_recon_config* cfg, const float* d_images, const double* params,
                                  long nparts, float* d_out, void* stream);

/* ---- projection matching (brefine's scoring path) -------------------------
 *
 *   bsg_match_create        <- project_refine_orientations' set-up
 *                              (bsoft/src/mg/mg_refine.cpp:279-316): resolution
 *                              checks, transform cut edge, FSI_Kernel
 *                              (bsoft/include/FSI_Kernel.h:28-68)
 *   bsg_match_set_reference <- pref->fft(), change_transform_size, clearing the
 *                              zero-frequency term, phase_shift_to_origin
 *                              (mg_refine.cpp:279-365)
 *   bsg_match_sections      <- Bimage::central_section (Bimage.h:995,
 *                              bsoft/src/img/Bimage_project.cpp:288-338) at the
 *                              resolution img_fit_in_recip_space_grid uses
 *                              (hi_res / 1.11, mg_refine.cpp:885)
 *   bsg_match_set_images    <- part_refine_orientation's particle preparation
 *                              (mg_refine.cpp:509-563)
 *   bsg_match_project       <- Bimage::project (Bimage.h:996,
 *                              bsoft/src/img/Bimage_project.cpp:362-443)
 *   bsg_match_score         <- one hypothesis of img_fit_in_recip_space_grid:
 *                              origin, phase_shift_to_origin, central_section,
 *                              img_recip_space_fom (mg_refine.cpp:660-781,
 *                              external linkage, no header in the reference)
 */
#define BSG_MATCH_APPLY_CTF  1   /* CTF record flag: multiply the reference by the CTF (APPLY_CTF) */
#define BSG_MATCH_INVERT     2   /* CTF record flag: contrast inversion (INVERT)                 */

/* Per-image CTF record, 8 doubles: volt, abw00, abw20, abw22, abw2m2, abw40,
 * flags (BSG_MATCH_*), 0.  As in img_recip_space_fom the CTF is applied only
 * when the defocus abw20 / (-pi lambda) is at least 1 angstrom. */
#define BSG_MATCH_CTF_DOUBLES 8
/* Hypothesis record, 12 doubles: image index, view matrix (row-major, as
 * View::matrix), origin x, y in pixels of the particle image. */
#define BSG_MATCH_HYP_DOUBLES 12

typedef struct {
    int    n;             /* particle box edge: power of two, 32..512           */
    int    map;           /* reference map edge N: power of two, 8..512         */
    double map_sampling;  /* angstrom / voxel of the reference map              */
    double pixel;         /* angstrom / pixel of the particle images            */
    double hi_res;        /* high resolution limit (angstrom)                   */
    double lo_res;        /* low resolution limit (angstrom), 0 = none          */
    int    kernel_width;  /* FSI kernel width (reference default 8, max 8)      */
    int    kernel_power;  /* FSI kernel power (reference default 2)             */
    int    batch;         /* images per device chunk, 0 = automatic             */
    int    device;        /* CUDA device ordinal                                */
} bsg_match_config;

typedef struct {
    int    diam;             /* edge of the cut transforms                      */
    int    npix;             /* pixels entering a figure of merit               */
    int    nshell;           /* shells kept                                     */
    double hi_res;           /* resolution after the reference's checks         */
    double max_rad;          /* FRC radius (pixels of the cut transform)        */
    double section_res;      /* central-section limit (hi_res / 1.11)           */
    double map_sampling_cut; /* sampling of the cut reference transform         */
    double pixel_cut;        /* sampling of the cut particle transforms         */
} bsg_match_info_t;

typedef struct bsg_match bsg_match;

int  bsg_match_create(const bsg_match_config* cfg, bsg_match** out);
void bsg_match_destroy(bsg_match* m);
int  bsg_match_info(const bsg_match* m, bsg_match_info_t* info);

/* Reference map (N^3 float32, x fastest) and its origin in voxels. */
int  bsg_match_set_reference(bsg_match* m, const float* map, const double* origin, int flags);
/* The prepared reference transform: diam^3 complex64, reference order. */
int  bsg_match_reference_transform(bsg_match* m, float* out, int flags);
/* Central sections for nviews row-major matrices: nviews x diam^2 complex64. */
int  bsg_match_sections(bsg_match* m, const double* mats, long nviews, float* out, int flags);
/* Projections (Bimage::project with the FSI kernel, Bimage.h:996,
 * bsoft/src/img/Bimage_project.cpp:362-443, back-transformed, real part):
 * nviews x N x N float32 of the UNCUT reference transform, pixels within
 * `resolution` (angstrom; <= 0: the sampling).  origins (nviews x 2 pixels,
 * NULL = N/2, the reference's phase_shift_to_center) place each projection;
 * ctf (nviews CTF records, NULL = none) multiplies each section by its CTF
 * first - an addition for synthesising particle images. */
int  bsg_match_project(bsg_match* m, const double* mats, long nviews, double resolution,
                       const double* origins, const double* ctf, float* out, int flags);
/* Particle images (nimg x n x n float32) with their CTF records; file_avg /
 * file_std are the statistics rescale_to_avg_std divides by (for a stack
 * read by the reference: the file header's), file_std <= 0 uses each
 * image's own.  Replaces the images held before. */
int  bsg_match_set_images(bsg_match* m, const float* images, long nimg, const double* ctf,
                          double file_avg, double file_std, int flags);
/* Prepared particle transforms [first, first+count): diam^2 complex64 each. */
int  bsg_match_prepared(bsg_match* m, long first, long count, float* out, int flags);
/* Figure of merit (and cross-validation figure) of nhyp hypotheses: the
 * FRC form (img_recip_space_fom fom_type 0), or with BSG_MATCH_SCORE_DPR the
 * DPR form (fom_type 1, brefine -fomtype dpr, mg_refine.cpp:725-772).
 * flags: BSG_MATCH_SCORE_FP64 gathers and sums in FP64 (the reference's
 * accumulation; ~1e-8 from its figures of merit, the FP32 default ~1e-7). */
#define BSG_MATCH_SCORE_FP64 4
#define BSG_MATCH_SCORE_DPR  8
int  bsg_match_score(bsg_match* m, const double* hyps, long nhyp, double* fom, double* cv, int flags);

/* Shell weights of the figure of merit (img_recip_space_fom's weight curve,
 * bsoft/src/mg/mg_refine.cpp:702-704): w[j] for shells j < n replaces the
 * unit weight where it is non-zero.  brefine always passes one:
 * project_refine_orientations uses C_curve(diam, 1 / (diam x cut sampling))
 * unless a curve is given (mg_refine.cpp:366-367, bsoft/src/util/
 * ctf.cpp:795-810).  n = 0 restores unit weights.  Applies to every later
 * scoring call (bsg_match_score, bsg_match_refine, the searches' exact
 * rescoring). */
int  bsg_match_set_shell_weights(bsg_match* m, const double* w, int n);

/* Exhaustive search (no counterpart in the reference, which refines locally
 * with img_refine_grid and scores with img_recip_space_fom; this is the
 * global search that scoring generalises to).
 *
 * bsg_match_set_panel: the search panel for nsec views (row-major matrices):
 * the central section of each at the coarse pixels (Hermitian half plane,
 * shells 1 .. ceil(max_rad) - 1), every shell normalised to unit power,
 * stored as BF16 (nsec x ~2 npix/2 x 2 bytes on the device).  Unless flags
 * has BSG_MATCH_PANEL_GATHER, the panel's FP32 sections at the
 * figure-of-merit pixels are kept too (nsec x npix x 8 bytes, when they fit
 * with 8 GB to spare): the exact rescoring then reads them instead of
 * gathering every candidate's section, with the same values.
 *
 * bsg_match_search: every held image at each of norigin trial origins
 * (origins: norigin x 2 doubles, pixels of the particle image) against every
 * panel section, by a BF16 correlation with FP32 accumulation on the tensor
 * cores: the per-shell FRC with the shell power of the CTF-weighted section
 * taken as (shell power of the section) x (shell mean of CTF^2).  The topk
 * best (section, origin) pairs of each image are rescored with the exact
 * figure of merit (bsg_match_score) and returned best first:
 * out = nimg x topk records of BSG_MATCH_RESULT_DOUBLES doubles:
 * section index, origin index, correlation score, FRC figure of merit,
 * cross-validation figure (section -1 if fewer candidates exist). */
#define BSG_MATCH_RESULT_DOUBLES 5
#define BSG_MATCH_TOPK_MAX 8
#define BSG_MATCH_PANEL_GATHER 1
int  bsg_match_set_panel(bsg_match* m, const double* mats, long nsec, int flags);
int  bsg_match_search(bsg_match* m, const double* origins, int norigin, int topk, double* out, int flags);
/* The same scoring restricted to the neighbourhood of a proposal per held
 * image (proposals: nimg x BSG_CNN_RESULT_FLOATS floats, host or with
 * BSG_DEVICE_PTR device: rotation row-major and shift from the box centre):
 * panel sections within `radius` (radians) of the proposed rotation and the
 * (at most 9) trial origins within origin_radius pixels of the proposed
 * origin, nearest first (the nearest is always kept).  At most 1,024
 * sections per image are considered.  Same output as bsg_match_search. */
int  bsg_match_search_local(bsg_match* m, const float* proposals, double radius, const double* origins, int norigin,
                            double origin_radius, int topk, double* out, int flags);

/* Device times of the search stages (CUDA events on the context's stream). */
typedef struct {
    double panel_ms;       /* panel construction                           */
    double agen_ms;        /* image rows (origin phase, CTF, shell norms)  */
    double gemm_ms;        /* tensor-core correlation with top-8 selection */
    double merge_ms;       /* per-image candidate merge                    */
    double rescore_ms;     /* exact figure of merit of the candidates      */
    double local_ms;       /* local search: selection and scoring          */
    double gemm_flops;     /* algorithmic: 2 x rows x sections x K         */
    double hypotheses;     /* image x origin x section triples scored      */
    long   launches;       /* kernels launched by the search calls         */
    long   gemm_launches;
    long   images;
    long   rescored;
    int    coarse_k;       /* real K of the correlation (2 x coarse pixels) */
    int    kpad;           /* K padded to the 64-element stage width        */
    double refine_ms;      /* grid refinement: figure-of-merit launches     */
    long   refine_launches;
    double panel_exact_ms; /* the panel's FP32 sections for the rescoring  */
    double panel_exact_bytes;  /* their device bytes (0: not kept)          */
} bsg_match_stats;
int  bsg_match_get_stats(bsg_match* m, bsg_match_stats* st);
int  bsg_match_reset_stats(bsg_match* m);
void* bsg_match_stream(bsg_match* m);        /* the context's cudaStream_t */

/* Grid refinement of orientations and origins: brefine without -monte, i.e.
 * img_refine_grid (bsoft/src/mg/mg_refine.cpp:1086-1195) with its shift
 * search img_fit_in_recip_space_grid (:862-950) and the view grid of
 * views_for_refinement (bsoft/src/util/View.cpp:371-424), for every start
 * record at once.  start: nstart records of BSG_MATCH_REFINE_START_DOUBLES
 * doubles: held image index, view x, y, z, angle (radians), origin x, y
 * (pixels of the particle image); an image may appear in several records
 * (part_refine_orientation refines from each symmetry-related view).
 * alpha_step, accuracy: angular step and final accuracy (radians; the
 * reference's checks: both >= 1e-30, step >= accuracy); shift_step,
 * shift_accuracy: origin grid step and accuracy (pixels of the cut
 * transform, as img_fit_in_recip_space_grid uses them; accuracy > 0).
 * def_std > 0 (angstrom): brefine -defocus: for every view the CTF is
 * applied at the 10 or 11 defoci d - 5 def_std .. d + 5 def_std around the
 * image's defocus d (its CTF record's abw20) at the original origin, and
 * the best of them is used for the view's shift grid (mg_refine.cpp:866-911,
 * 1105-1191); every held image needs a voltage and a non-zero defocus.
 * def_std = 0: the held images' CTF records apply as set_images gave them
 * (in the reference the grid refinement applies a CTF only with -defocus).
 * out: nstart records of BSG_MATCH_REFINE_RESULT_DOUBLES doubles: view x,
 * y, z, angle, origin x, y (pixels of the particle image), figure of merit,
 * cross-validation figure, hypotheses scored (the reference's `number`),
 * defocus after refinement (angstrom; 0 without the defocus search),
 * particle pixel size x, y after refinement (angstrom: the refined sampling
 * of the cut transform times the cut scale, part_refine_orientation,
 * mg_refine.cpp:633).
 * max_mag in (0, 1): brefine -magnification: after the angular rounds,
 * img_refine_grid's magnification stage (mg_refine.cpp:1145-1187) fits the
 * best view at every pair of per-axis sampling factors 1 - max_mag ..
 * 1 + max_mag (steps max_mag / 10, y outer; 441 pairs) with shift steps
 * 0.4 -> 0.1 around the best origin, and keeps the best fit; 0: none.
 * flags: BSG_MATCH_SCORE_DPR scores with the DPR figure of merit (brefine
 * -fomtype dpr). */
#define BSG_MATCH_REFINE_START_DOUBLES 7
#define BSG_MATCH_REFINE_RESULT_DOUBLES 12
int  bsg_match_refine(bsg_match* m, const double* start, long nstart, double alpha_step, double accuracy,
                      double shift_step, double shift_accuracy, double def_std, double max_mag, double* out,
                      int flags);

/* brefine -monte: Monte Carlo refinement, img_refine_monte (bsoft/src/mg/
 * mg_refine.cpp:979-1050) with img_fit_in_recip_space_monte (:783-860), for
 * every start record (layout as bsg_match_refine's).  max_iter outer
 * iterations perturb the view (vector3_random_gaussian of view_std, an
 * in-plane step of up to max_angle radians, per-axis sampling factors 1 +-
 * max_mag), each fitted by max_iter inner iterations that perturb the
 * origin (shift_std, pixels of the cut transform) and, with def_std > 0
 * (angstrom), the defocus; steps are accepted when fom / previous fom
 * exceeds a uniform draw.  The random numbers are the C library's random()
 * after srandom(seed) (the reference seeds with its process id), drawn
 * record after record in the reference's order, so a seed reproduces the
 * reference's run; seed 0 continues the context's stream from the previous
 * call (a run split into batches draws one sequence).  out: as
 * bsg_match_refine's (hypotheses = max_iter^2). */
int  bsg_match_refine_monte(bsg_match* m, const double* start, long nstart, int max_iter, double def_std,
                            double shift_std, double view_std, double max_angle, double max_mag,
                            unsigned long long seed, double* out, int flags);

/* ---- learned orientation proposer ------------------------------------------
 * No counterpart in the reference.  A convolutional network maps a particle
 * image to a rotation and a shift; bsg_match_search_local then searches
 * only the panel sections near each proposal.  6 convolutions (3x3, stride
 * 2, ReLU), two dense layers, a 6-D rotation head (Gram-Schmidt); weights
 * held in FP32, used rounded to BF16, FP32 accumulation.
 * Parameter order: for each convolution W[cout][3][3][cin], b[cout]; then
 * fc1 W[hidden][(box/64)^2 * c6] (input flattened y, x, channel), b; fc2
 * W[8][hidden], b.  Outputs per image (BSG_CNN_RESULT_FLOATS): rotation
 * matrix row-major (9, columns b1 b2 b3), shift x, y (pixels from the box
 * centre). */
#define BSG_CNN_RESULT_FLOATS 11
typedef struct {
    int    box;            /* image edge: power of two, 64..512             */
    int    channels[6];    /* output channels of the 6 convolutions         */
    int    hidden;         /* width of the dense layer                      */
    int    batch;          /* mini-batch (training) / chunk (inference)     */
    float  shift_weight;   /* lambda of the shift term of the loss          */
    int    device;
    unsigned long long seed;   /* initialisation and batch sampling         */
} bsg_cnn_config;

typedef struct bsg_cnn bsg_cnn;

int  bsg_cnn_create(const bsg_cnn_config* cfg, bsg_cnn** out);
void bsg_cnn_destroy(bsg_cnn* c);
long bsg_cnn_num_params(const bsg_cnn* c);
int  bsg_cnn_get_params(bsg_cnn* c, float* out);
int  bsg_cnn_set_params(bsg_cnn* c, const float* in);      /* resets the optimiser */
/* n images (box^2 float32 each) -> n x BSG_CNN_RESULT_FLOATS */
int  bsg_cnn_predict(bsg_cnn* c, const float* images, long n, float* out, int flags);
/* mean loss and its gradient (all parameters) for n host images with host
 * targets (n x BSG_CNN_RESULT_FLOATS: true rotation and shift) */
int  bsg_cnn_loss_grad(bsg_cnn* c, const float* images, const float* targets, long n, double* loss, float* grads);
/* `steps` Adam steps on mini-batches drawn without replacement from ndata
 * device-resident images and targets (BSG_DEVICE_PTR required); losses
 * (host, optional) receives the mean loss of each step */
int  bsg_cnn_train(bsg_cnn* c, const float* images, const float* targets, long ndata, int steps, float lr,
                   float* losses, int flags);

/* Data synthesis: Gaussian noise added to n device images (box^2 each) at a
 * signal-to-noise ratio relative to each image's variance inside the
 * inscribed circle; counter-based, reproducible for a seed. */
int  bsg_add_noise(float* d_images, long n, int box, double snr, unsigned long long seed, void* stream);

/* ---------------------------------------------------------------------------
 * Real-space weighted back-projection (bbackproj).
 *
 *   bsg_backproj_create  <- the map set-up of project_back_projection
 *                           (bsoft/src/mg/mg_reconstruct.cpp:1524-1560) and the
 *                           plans of bbackproj (bsoft/src/bbackproj.cpp:170-171)
 *   bsg_backproj_add     <- its per-particle loop (mg_reconstruct.cpp:1570-1614)
 *                           over Bimage::back_project (bsoft/src/img/
 *                           Bimage_project.cpp:466-509): ramp filter
 *                           (fspace_weigh_ramp), rescale to average 0 and
 *                           standard deviation 1, background fill, every voxel
 *                           adds the image sampled along its projection
 *   bsg_backproj_finish  <- img_backprojection_accumulate (mg_reconstruct.cpp:
 *                           1640-1684) and bbackproj's -symmetry / -rescale
 *                           (bbackproj.cpp:199-207)
 *
 * Record per image: BSG_BACKPROJ_DOUBLES doubles
 *   [0..1]  image origin x, y (pixels)      Bparticle::ori as project_back_
 *                                           projection resolves it
 *   [2..10] rotation matrix, row-major      View::matrix (View.h:153-156)
 *   [11]    magnification (part->mag / scale; > 0)
 *   [12]    map index: 0, or 1 for the second half map
 *   [13]    image pixel size (angstrom; 0: the config's), which sets the
 *           ramp's frequencies and resolution check (Bparticle::pixel_size)
 *   [14..15] reserved (0)
 * The map is N^3 float32, z slowest, origin at its integer half size.
 */
#define BSG_BACKPROJ_DOUBLES 16

typedef struct {
    int    n;             /* image edge (square images), 2..1024 with no    */
                          /* prime factor above 7                           */
    int    map;           /* map edge N, 2..1024                            */
    double pixel;         /* image pixel size (angstrom) of records with 0  */
    double resolution;    /* ramp limit (angstrom), checked per image as    */
                          /* Bimage::check_resolution does                  */
    int    nmaps;         /* 1 full map; 2 (or 3) two half maps as well     */
    int    batch;         /* images per device batch (0: 256)               */
    int    device;
} bsg_backproj_config;

typedef struct bsg_backproj bsg_backproj;

int  bsg_backproj_create(const bsg_backproj_config* cfg, bsg_backproj** out);
void bsg_backproj_destroy(bsg_backproj* b);
/* count images (n^2 float32 each, host, or device with BSG_DEVICE_PTR) and
 * their records; the map(s) grow in image order.  Returns when the inputs
 * may be reused. */
int  bsg_backproj_add(bsg_backproj* b, const float* images, const double* records, long count, int flags);
/* Map imap (0: the full map, the float sum of the halves when there are
 * two; 1, 2: a half map), after the optional symmetrization and rescaling,
 * into map_out (N^3 float32; a device pointer with BSG_DEVICE_PTR). */
int  bsg_backproj_finish(bsg_backproj* b, int imap, float* map_out, int flags);
/* bbackproj -symmetry: Bimage::symmetrize(sym, 1) of the finished map
 * (generating operations as bsg_recon_set_symmetrize takes them); nops 0
 * turns it off. */
int  bsg_backproj_set_symmetrize(bsg_backproj* b, const double* axes, const int* orders, int nops);
/* bbackproj -rescale avg,std (std <= 0: off) */
int  bsg_backproj_set_rescale(bsg_backproj* b, double avg, double std);
int  bsg_backproj_reset(bsg_backproj* b);

const char* bsg_last_error(void);
const char* bsg_version(void);

#ifdef __cplusplus
}
#endif

#endif
