/*
 * oracle.h - FP64 CPU restatement of the reference's single-particle
 * reconstruction and projection-matching path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this; it
 * is the checker that the CUDA path is compared against (tests/, the smoke
 * check and the CPU-baseline leg of bench.py).  Every function cites the
 * reference lines it restates.  The restatement itself is pinned against
 * the reference's own programs compiled from source (oracle/_ref) through
 * the fixtures under tests/golden/.
 */
#ifndef BSOFT_ORACLE_H
#define BSOFT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Reconstruction geometry shared by all particles of a run. */
typedef struct {
    int    n;            /* particle box edge (images are n x n)            */
    int    ft;           /* padded transform edge (part_ft_size)            */
    int    map;          /* map edge N                                      */
    double map_sampling; /* angstrom / voxel of the map                     */
    double hi_res;       /* resolution limit after Bimage::check_resolution */
    int    interp;       /* 0 nearest, 1 weighted nearest, 2 trilinear      */
    int    ctf_action;   /* 0 none, 1 flip, 2 apply, >=3 Wiener-type        */
    double wiener;       /* Wiener factor (0 -> plain multiply unless flip)  */
} orc_recon_cfg;

/* Per-particle parameters (host-prepared, see bsoft_b200/recon.py). */
typedef struct {
    double origin[2];     /* particle origin, pixels                         */
    double bkg_center[2]; /* centre of the background circle (file origin)   */
    double mat[9];        /* view rotation matrix, row-major                 */
    double pixel;         /* particle pixel size, angstrom                   */
    double scale;         /* 1/magnification (1 if none)                     */
    double weight;        /* particle weight (1, or selection for bootstrap) */
    double ctf[7];        /* abw00 abw20 abw22 abw2m2 abw40 abw11 abw1m1     */
    double ewald;         /* electron wavelength (angstrom) for Ewald-sphere
                             insertion (breconstruct -ewald), 0 = plane      */
} orc_particle;

/* Accumulate particles into FP64 volumes: vol (2*N^3, complex), weight
 * (N^3); power and weight2 (N^3) may be NULL.  Returns 0 or <0 on error. */
int orc_insert(const orc_recon_cfg* cfg, const float* images, const orc_particle* parts,
               long nparts, double* vol, double* weight, double* power, double* weight2);

/* One particle's transform after pad, FFT, origin shift and CTF:
 * out = ft*ft complex doubles.  Used to check the 2-D stage on its own. */
int orc_particle_transform(const orc_recon_cfg* cfg, const float* image,
                           const orc_particle* part, double* out);

/* Weigh, shift to centre, inverse 3-D FFT (1/sqrt(N^3)), real part and, when
 * sinc != 0, the trilinear sinc compensation.  vol/weight are modified in
 * place; map_out receives N^3 floats.  Returns coverage (voxels weighed). */
long orc_finish(const orc_recon_cfg* cfg, double* vol, double* weight, double* power,
                double* weight2, double* map_out, int sinc);

/* FSC of two complex N^3 transforms as Bimage::fsc(Bimage*) forms it
 * (linearly interpolated shells, sampling ratio 1, shells below
 * real_size / hi_res): nshell values, FSC[0] = 1.  Returns the shell count. */
int orc_fsc(int N, const double* vol1, const double* vol2, double real_size, double hi_res, int nshell, double* fsc);

/* ---- projection matching (match_oracle.c) ---- */

/* FSI_Kernel lookup table: (512 + 1) * width doubles.  Returns the width
 * actually used (1 for a negative power) or <0. */
int orc_fsi_kernel(int width, int power, double* table);

/* Transform edge the reference map is cut to for a resolution limit. */
int orc_match_diam(int N, double sampling, double hi_res);

/* Reference map (real N^3, z-y-x order) -> its transform cut to diam^3
 * (standard layout, 2*diam^3 doubles), zero-frequency term cleared, phase
 * shifted to origin*diam/N.  spec must hold 2*N^3 doubles. */
int orc_match_map(int N, const float* map, const double origin[3], double sampling, double hi_res,
                  double* spec, int* diam_out);

/* Kernel interpolation of a complex size^3 transform at voxel position m. */
void orc_fspace_interpolate(int size, const double* spec, const double m[3], const double* kernel, int wd,
                            double out[2]);

/* Central section (size^2 complex doubles) of a size^3 transform for the
 * row-major rotation `mat`, real_size = size * sampling (angstrom), pixels
 * with s <= 1/resolution only. */
int orc_central_section(int size, const double* spec, const double* mat, double real_size, double resolution,
                        const double* kernel, int wd, double* out);

/* Particle image (n^2 floats) -> transform of (image - avg)/std, unscaled,
 * cut to diam^2 (2*diam^2 doubles), zero-frequency term cleared.  avg/std
 * are the stack file's statistics (std <= 0: this image's own). */
int orc_match_particle(int n, const float* image, int diam, double file_avg, double file_std, double* spec);

/* In-place phase shift of a size^2 transform to an origin in pixels. */
void orc_phase_shift_2d(int size, double* spec, const double origin[2]);

/* img_recip_space_fom: FRC (fom_type 0) or DPR (1) figure of merit of an
 * image transform against a reference section, both size^2 complex; ctf is
 * NULL or the 7 aberration weights (the reference section is multiplied by
 * the CTF, negated when invert).  The cross-validation figure goes to
 * *cv_out. */
double orc_recip_space_fom(int size, const double* img, const double* ref, double img_real_size,
                           double ref_real_size, double ref_sampling, double hi_res, double lo_res,
                           int fom_type, const double* ctf, int invert, double* cv_out);

#ifdef __cplusplus
}
#endif

#endif
