// common.cuh - shared definitions of the sm_100a reconstruction library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/bsgpu.h"

namespace bsg {

void set_error(const char* fmt, ...);

#define BSG_CHECK_CUDA(call)                                                       \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            ::bsg::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                             __FILE__, __LINE__);                                  \
            return BSG_ERR_CUDA;                                                   \
        }                                                                          \
    } while (0)

// Per-particle record as the device kernels read it.  Built on the host
// from the 32-double C-ABI record (bsgpu.h) and the run geometry.
struct alignas(16) DevParticle {
    // 2-D stage
    double shx, shy;        // phase-shift slope: 2*pi*origin/ft (Bimage_complex.cpp:510)
    double bx, by;          // background circle centre (pixels)
    double fs;              // CTF frequency step 1/(ft*pixel)   (mg_ctf.cpp:84-85)
    double c00, c20, c22, c2m2, c40, c11, c1m1;   // aberration weights (ctf.h:321-348)
    // insertion (fspace_pack_2D, Bimage_reconstruct.cpp:131-160)
    double ad[3], bd[3];    // map frequency per unit pixel step: R[:,0]*inv*mscale, R[:,1]*inv*mscale
    double iad[3], ibd[3];  // 1 / ad, 1 / bd (0 where |.| <= 1e-12): the gridding walks' row and line bounds
    double nrm[3];          // unit plane normal R[:,2]
    double inv2;            // (scale/(ft*pixel))^2: s2 per unit pixel^2
    double inv_st2;         // 1 / step^2: pixel coordinate per unit of ad.c
    double na, nb;          // image normalisation v * na + nb (breconstruct -rescale; 1, 0 otherwise)
    // Ewald-sphere surface (breconstruct -ewald; Bimage_reconstruct.cpp:157-168):
    // m += ewh s2 cd with s2 = (h^2 + k^2) inv2, one record per surface
    double ewh;             // +-lambda/2 (0: the plane)
    double inv;             // sqrt(inv2): s per unit pixel
    double cd[3];           // R[:,2] * mscale
    float  ezmax;           // max |ewh s2| mscale over the pixels (voxels)
    float  ib[3];           // 1 / bf[i] (0 when |bf[i]| <= 1e-6)
    float  inv_step;        // 1 / step
    float  af[3], bf[3];    // float copies of ad / bd
    float  pw;              // particle weight / (pad_ratio^2 * 0.6)
    float  slab;            // sum |nrm_i|: plane reaches a voxel cube iff |n.c| < slab
    float  step;            // |ad| = voxels per pixel step
    int    half;            // half-map index
    int    spec;            // index of this record's spectrum in the batch (symmetry copies share it)
    int    lat;             // gridding phase lattice lh | lk << 12 | sh << 24 (lattice.h); 0: the
                            // orientation-independent one
};

// Run geometry shared by all kernels of one context.
struct Geometry {
    int n, ft, map, logft;
    int interp, ctf_action;
    double wiener;
    double hi_res;          // insertion limit (>= 0.5, Bimage_reconstruct.cpp:136)
    double maxs2, mins2;    // insertion s^2 window
    double ctf_shi2;        // CTF s^2 upper limit (mg_ctf.cpp:50-60)
    double mscale;          // map real size N * sampling
    int    fom;
    int    gate;           // 1: some pixel may fall outside the s^2 window or in the taper
    int    ewald;          // 1: the batch's records include Ewald-sphere surfaces
};

__host__ __device__ inline int ilog2i(int v) { int l = 0; while ((1 << l) < v) ++l; return l; }

// signed frequency of index i along an axis of length L (Bimage convention:
// i > (L-1)/2 -> i - L)
__host__ __device__ inline int sfreq(int i, int L) { return i > (L - 1) / 2 ? i - L : i; }

struct Context;

// kernels launchers (return cudaError_t of the launch)
cudaError_t launch_background(const Context& c, const float* img, int nimg, cudaStream_t s);
cudaError_t launch_rows(const Context& c, const float* img, int nimg, cudaStream_t s);
cudaError_t launch_cols(const Context& c, int nimg, float2* spectra, cudaStream_t s);
cudaError_t launch_insert(const Context& c, const float2* spectra, const DevParticle* parts, int np, int half,
                          cudaStream_t s);
cudaError_t launch_finish(const Context& c, int imap, float* map_out, float* fom_out, bool sinc, cudaStream_t s);
cudaError_t launch_fsc(const Context& c, int nshell, double* out_dev, cudaStream_t s);
cudaError_t launch_symmetrize(const Context& c, float* map, float* tmp, bool sinc, cudaStream_t s);
cudaError_t launch_rescale(const Context& c, float* map, double nuavg, double nustd, bool sinc, cudaStream_t s);

}  // namespace bsg
