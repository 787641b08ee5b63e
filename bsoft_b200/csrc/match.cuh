// match.cuh - the projection-matching context shared by match.cu (transforms,
// sections, exact scoring) and search.cu (the exhaustive BF16 search).
#pragma once

#include "common.cuh"

#include <cuda_bf16.h>

#include <stdlib.h>

#include <vector>

namespace bsg {

constexpr int NDIV = 512;     // FSI_Kernel divisions (FSI_Kernel.h:42)
constexpr int MAXW = 8;       // widest kernel the warp gather supports
constexpr int FOM_WARPS = 8;

struct MPix {
    short h, k;     // signed frequency indices
    int idx;        // index in the diam^2 transform
    short shell;    // (long) sqrt(h^2 + k^2)
    short insec;    // 1: inside the section's resolution limit
    int pad;
};
static_assert(sizeof(MPix) == 16, "MPix layout");

constexpr int MAXORG = 9;     // trial origins scored per gathered section

struct MHyp {
    double m[9];    // view matrix with rows 0, 1 scaled (mg_refine.cpp:876-880)
    double sx, sy;  // phase slopes 2 pi origin / diam (cut pixels)
    int img;
    int pad;
};

// one image and view with up to MAXORG origins (the exact figure of merit
// gathers the section once and scores every origin from it)
struct MHypG {
    double m[9];
    double sx[MAXORG], sy[MAXORG];
    int img;
    int norg;
    int ctf;        // row of the CTF table the launch scores with (the image's own: img)
    int sec;        // gathered section of the launch's section buffer (when it has one)
};


__device__ __forceinline__ int wrap1(int j, int D) {
    if (j < 0) j += D;
    if (j >= D) j -= D;
    // only reachable for positions more than a map edge outside, which the
    // reference would read out of bounds: keep the access inside
    return min(max(j, 0), D - 1);
}

// Sources of the cut reference transform for the gather: the linear array
// (reference index order) or a 3-D texture over the same values.  The
// texture's block-linear layout keeps an 8^3 tap neighbourhood on far fewer
// cache lines than z-major rows, which is what limits the gather when many
// warps work on different rotations at once.
struct PtrSrc {
    const float2* __restrict__ p;
    int D;
    __device__ __forceinline__ float2 operator()(int x, int y, int z) const {
        return __ldg(p + ((size_t)z * D + y) * D + x);
    }
};
struct TexSrc {
    cudaTextureObject_t t;
    __device__ __forceinline__ float2 operator()(int x, int y, int z) const {
        return tex3D<float2>(t, (float)x, (float)y, (float)z);
    }
};

// FSI kernel interpolation of the diam^3 transform at voxel position m by
// one warp (Bimage::fspace_interpolate).  Every lane returns the sum.
// T = double (with an FP64 kernel table) accumulates as the reference does;
// T = float agrees with it to ~1e-8 in the figure of merit (the transforms
// themselves are computed in FP64, which is what the outer shells need).
template <typename T, typename Src>
__device__ __forceinline__ void fsi_gather_any(const Src& src, int D, double mx, double my, double mz,
                                           const T* __restrict__ lut, int wd, int lane, T& out_re, T& out_im) {
    const int half = (wd - 1) / 2;
    const double fx = floor(mx), fy = floor(my), fz = floor(mz);
    const int ikx = (int)((mx - fx) * NDIV + 0.5) * wd;
    const int iky = (int)((my - fy) * NDIV + 0.5) * wd;
    const int ikz = (int)((mz - fz) * NDIV + 0.5) * wd;
    const int ibx = (int)fx - half, iby = (int)fy - half, ibz = (int)fz - half;
    const int xl = lane & 7, rq = lane >> 3;
    T ar = 0, ai = 0;
    if (xl < wd) {
        const int jx = wrap1(ibx + xl, D);
        const T kx = lut[ikx + xl];
        for (int r = rq; r < wd * wd; r += 4) {
            const int zz = r / wd, yy = r - zz * wd;
            const int jz = wrap1(ibz + zz, D), jy = wrap1(iby + yy, D);
            const T w = kx * (lut[iky + yy] * lut[ikz + zz]);
            const float2 v = src(jx, jy, jz);
            ar += (T)v.x * w;
            ai += (T)v.y * w;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        ar += __shfl_xor_sync(0xffffffffu, ar, o);
        ai += __shfl_xor_sync(0xffffffffu, ai, o);
    }
    out_re = ar;
    out_im = ai;
}

// The reference's default width 8: lane = (x tap, row group rq); the lane's
// rows are y = rq and rq + 4 at every z, so the wraps and the y weights are
// computed once and the z loop unrolls.  Same taps, weights and summation
// order as fsi_gather_any.
template <typename T, typename Src>
__device__ __forceinline__ void fsi_gather8(const Src& src, int D, double mx, double my, double mz,
                                            const T* __restrict__ lut, int lane, T& out_re, T& out_im) {
    const double fx = floor(mx), fy = floor(my), fz = floor(mz);
    const int ikx = (int)((mx - fx) * NDIV + 0.5) * 8;
    const int iky = (int)((my - fy) * NDIV + 0.5) * 8;
    const int ikz = (int)((mz - fz) * NDIV + 0.5) * 8;
    const int ibx = (int)fx - 3, iby = (int)fy - 3, ibz = (int)fz - 3;
    const int xl = lane & 7, rq = lane >> 3;
    const int jx = wrap1(ibx + xl, D);
    const int jy0 = wrap1(iby + rq, D), jy1 = wrap1(iby + rq + 4, D);
    const T kx = lut[ikx + xl], ky0 = lut[iky + rq], ky1 = lut[iky + rq + 4];
    T ar = 0, ai = 0;
#pragma unroll
    for (int z = 0; z < 8; ++z) {
        const int jz = wrap1(ibz + z, D);
        const T kz = lut[ikz + z];
        const float2 v0 = src(jx, jy0, jz);
        const float2 v1 = src(jx, jy1, jz);
        const T wa = kx * (ky0 * kz), wb = kx * (ky1 * kz);
        ar += (T)v0.x * wa;
        ai += (T)v0.y * wa;
        ar += (T)v1.x * wb;
        ai += (T)v1.y * wb;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        ar += __shfl_xor_sync(0xffffffffu, ar, o);
        ai += __shfl_xor_sync(0xffffffffu, ai, o);
    }
    out_re = ar;
    out_im = ai;
}

template <typename T, typename Src>
__device__ __forceinline__ void fsi_gather(const Src& src, int D, double mx, double my, double mz,
                                           const T* __restrict__ lut, int wd, int lane, T& out_re, T& out_im) {
    if (wd == 8) fsi_gather8<T, Src>(src, D, mx, my, mz, lut, lane, out_re, out_im);
    else fsi_gather_any<T, Src>(src, D, mx, my, mz, lut, wd, lane, out_re, out_im);
}

struct ImgCtf {
    double c[5];     // abw00 abw20 abw22 abw2m2 abw40
    int apply;       // multiply the reference by the CTF
    int invert;      // negate the CTF (contrast inversion)
    double fsx, fsy; // frequency per index on x and y (1 / real size of the image
                     // with its per-axis sampling); 0: the context's isotropic step
};

// sin(chi) of one figure-of-merit pixel (img_recip_space_fom's CTF factor,
// mg_refine.cpp:700-740; chi as CTFparam::calculate_aberration_even,
// ctf.h:321-334); 1 when the record does not apply
__device__ __forceinline__ float ctf_factor(const ImgCtf& C, const MPix& q, double fs) {
    if (!C.apply) return 1.f;
    double sx2 = (C.fsx > 0 ? C.fsx : fs) * q.h; sx2 *= sx2;
    double sy2 = (C.fsy > 0 ? C.fsy : fs) * q.k; sy2 *= sy2;
    const double s2 = sx2 + sy2;
    const double a = atan2((double)q.k, (double)q.h);
    const double chi = C.c[0] + s2 * (C.c[3] * sin(2 * a) + C.c[1] + C.c[2] * cos(2 * a)) + s2 * s2 * C.c[4];
    double s = sin(chi);
    if (C.invert) s = -s;
    return (float)s;
}

struct Match {
    bsg_match_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    int N = 0, n = 0, D = 0, wd = 8;
    double hi_res = 0, map_samp_cut = 0, img_samp_cut = 0, sec_res = 0;
    double real_map = 0, real_img = 0, max_rad = 0, max_rad_cv = 0;
    double scx = 1, scy = 1;           // pref sampling / particle sampling
    double cut_scale = 1;              // diam / n (long double in the reference)
    int nshell = 0, nf = 0, cv0 = 0, cv1 = 0;
    // per-shell weights of the figure of merit (img_recip_space_fom's w[j]:
    // 1, or the caller's curve where it is non-zero) and their sums over the
    // FRC shells [0, nf) and the cross-validation shells [cv0, cv1)
    // brefine -monte's random() stream (glibc random_r on a private TYPE_3
    // state), kept between calls so that batches continue one sequence
    random_data rng_data;
    char rng_state[128];
    bool rng_init = false;
    std::vector<double> h_wshell;
    double* d_wshell = nullptr;
    double wf = 0, wc = 0;
    std::vector<MPix> h_pix;           // figure-of-merit pixels, shell-sorted
    std::vector<int> h_shell_start;
    std::vector<MPix> h_secpix;        // section pixels
    MPix* d_pix = nullptr;
    int* d_shell_start = nullptr;
    MPix* d_secpix = nullptr;
    double* d_lut = nullptr;           // FSI table, FP64 (sections output)
    float* d_lutf = nullptr;           // FSI table, FP32 (scoring and search panel)
    double2* d_tw_map = nullptr;
    double2* d_tw_img = nullptr;
    float2* d_ref = nullptr;           // diam^3
    float2* d_full = nullptr;          // uncut N^3 transform for the projector
    cudaArray_t ref_array = nullptr;   // the same values behind a 3-D texture
    cudaTextureObject_t ref_tex = 0;
    bool have_ref = false;
    // images
    long cap = 0, nimg = 0;
    float2* d_spec = nullptr;          // cap x diam^2
    float* d_ctf = nullptr;            // cap x npix
    double* d_dsum = nullptr;          // cap x nshell
    // scratch
    float* d_real = nullptr;           // batch x n^2 (or N^3 for the map)
    double2* d_work = nullptr;         // batch x n^2 complex (or N^3), FP64
    size_t work_elems = 0;
    double* d_scale = nullptr;
    double* d_shift = nullptr;
    ImgCtf* d_ictf = nullptr;
    std::vector<ImgCtf> h_ictf;        // host copy of the held images' CTF records
    std::vector<double> h_volt;        // and their accelerating voltages
    MHyp* d_hyp = nullptr;
    long hyp_cap = 0;
    double* d_out = nullptr;           // 2 x hyp_cap
    MHypG* d_grp = nullptr;            // hypothesis groups for the exact score
    double* d_gout = nullptr;          // 2 x MAXORG x grp_cap
    long grp_cap = 0;
    float* h_pin = nullptr;            // pinned staging
    size_t pin_bytes = 0;
    // exhaustive search (search.cu)
    std::vector<MPix> h_cpix;          // coarse pixels: half plane, shells 1 .. nf-1
    std::vector<int> h_cstart;
    int ncpix = 0, kpad = 0;
    MPix* d_cpix = nullptr;
    int* d_cstart = nullptr;
    long nsec = 0;
    MHyp* d_secs = nullptr;            // panel views (rows 0, 1 scaled)
    std::vector<MHyp> h_secs;          // host copy
    float* d_rots = nullptr;           // panel rotations (unscaled, float) for local selection
    __nv_bfloat16* d_panel = nullptr;  // nsec x kpad
    float2* d_pexact = nullptr;        // nsec x npix: the panel's FP32 sections at the figure-of-merit
                                       // pixels, as fom_kernel<float> gathers them (rescoring reads them)
    __nv_bfloat16* d_A = nullptr;      // rows x kpad
    size_t a_elems = 0;
    float* d_pscore = nullptr;         // partial top-8 per (range, row)
    int* d_pidx = nullptr;
    size_t part_elems = 0;
    int* d_csec = nullptr;             // candidates per image
    int* d_corg = nullptr;
    float* d_cscore = nullptr;
    size_t cand_elems = 0;
    float* d_gA = nullptr;             // per image and shell: 1 / (n_f sqrt(D_j C_j))
    size_t gA_elems = 0;
    double2* d_slopes = nullptr;       // per trial origin
    size_t slope_elems = 0;
    int* d_status = nullptr;
    // local search scratch (grow-only)
    float* d_lprop = nullptr;          // nimg x 11 proposals
    int* d_lorg = nullptr;             // nimg x LOCAL_MAXO trial origins
    int* d_nlorg = nullptr;            // nimg
    long lscr_img = 0;
    int* d_lcand = nullptr;            // batch x LOCAL_MAXC selected sections
    int* d_lcount = nullptr;           // batch
    long lscr_nb = 0;
    bsg_match_stats sstats{};
};


// exact scoring of ng hypothesis groups already on the device (match.cu):
// d_fom / d_cv get MAXORG slots per group; fp64: FP64 gather and sums; dpr:
// the DPR figure of merit instead of the FRC
cudaError_t launch_fom(const Match& M, const MHypG* d_groups, long ng, double* d_fom, double* d_cv, cudaStream_t s,
                       bool fp64 = false, const float* ctf_table = nullptr, const double2* sec = nullptr,
                       bool dpr = false, const float2* psec = nullptr);
// FP32 sections of nsec panel views at the figure-of-merit pixels, gathered
// as fom_kernel<float> gathers them: nsec x npix float2 (0 where a pixel is
// outside the section)
cudaError_t launch_panel_exact(const Match& M, const MHyp* d_secs, long nsec, float2* d_out, cudaStream_t s);
// FP64 section values of nv views (9 doubles each, MHyp's scaled rows) at
// the figure-of-merit pixels: nv x npix double2
cudaError_t launch_secgather(const Match& M, const double* d_mats, long nv, double2* d_out, cudaStream_t s);
// CTF table rows (npix floats each) for nrec records on the device
cudaError_t launch_ctf_rows(const Match& M, const ImgCtf* d_rec, long nrec, float* d_out, cudaStream_t s);
void group_hypotheses(const std::vector<MHyp>& hyps, std::vector<MHypG>& groups, std::vector<long>& slot);
int ensure_groups(Match& M, long ng);
// view matrix rows 0, 1 scaled by the sampling ratio (img_fit_in_recip_space_grid)
void match_view_rows(const Match& M, const double* mat, double* m);
int match_fail(int code, const char* fmt, ...);

}  // namespace bsg
