// context.cuh - the state behind an opaque bsg_recon handle.
#pragma once

#include "common.cuh"

#include <cuda.h>

#include <vector>

namespace bsg {

struct Context {
    bsg_recon_config cfg;
    Geometry g;
    int device = 0;
    int batch = 0;
    int nhalves = 1;
    cudaStream_t stream = nullptr;

    // per-batch device buffers
    DevParticle* d_part = nullptr;   // batch (the current batch's buffer)
    // point-group symmetry (fspace_pack_2D over symmetry_get_all_views):
    // nsym operators S (row-major); particle records are gridded once per
    // operator with matrix S R, all copies reading the particle's spectrum
    std::vector<double> sym;          // 9 per operator; empty = C1
    DevParticle* d_psym = nullptr;    // batch x nsym expanded records (current batch)
    std::vector<DevParticle> h_psym;
    // point-group symmetrization after reconstruction (mode 1): generating
    // operations (axis as given, order), applied to the finished real map
    std::vector<double> symz_axes;    // 3 per operation
    std::vector<int> symz_orders;
    float* d_symtmp = nullptr;        // N^3 float work map
    double rescale_avg = 0, rescale_std = 0;   // -rescale (std > 0: on)
    double* d_bkg = nullptr;         // batch
    float2* d_phase = nullptr;       // batch x 2 x ft: exp(i h shx), exp(i k shy)
    float2* d_rows = nullptr;        // batch x n x (ft/2+1): row transforms
    float2* d_spec = nullptr;        // batch x (ft+1) x (ft+2): centred, padded particle spectra (current batch)
    float2* d_tw = nullptr;          // ft/2 twiddles exp(-2 pi i j / ft)
    float2* d_twmap = nullptr;       // N/2 twiddles exp(-2 pi i j / N)

    // accumulators per half map, reference index order, FP64 (each batch's
    // per-voxel sums are folded in once, so the long reduction over the
    // whole particle set is carried in double precision)
    double2* d_vol[2] = {nullptr, nullptr};
    double* d_w[2] = {nullptr, nullptr};
    double* d_pow[2] = {nullptr, nullptr};
    double* d_w2[2] = {nullptr, nullptr};

    // finishing buffers (allocated on first use)
    float2* d_work = nullptr;        // N^3 complex
    float* d_map = nullptr;          // N^3 real
    float* d_fom = nullptr;          // N^3 real
    float2* d_half_weighed[2] = {nullptr, nullptr};
    double* d_fsc = nullptr;         // FSC partial sums

    int shape = 0;                   // gridding tile shape (insert.cu kShapes)
    int* d_tile_order = nullptr;     // tile visiting order for `shape`
    int replicas = 1;                // warps per tile, each on a slice of the particles
    // half-space gridding (insert.cu, walk_edges): > 0 when the accumulators
    // below zsplit hold the paired pixels' sums (their unpaired pixels' sums
    // in d_evol / d_ew) and those at or above it the unpaired pixels' sums,
    // the rest being the conjugate of the mirrored voxels; 0: full map
    int zsplit = 0;
    bool half_space = true;          // allowed (bsg_recon_set_half_space)
    bool ewald_seen = false;         // an Ewald batch was gridded: full map for good
    bool dirty = false;              // something was inserted since the last reset
    double2* d_evol[2] = {nullptr, nullptr};   // half-space: unpaired pixels' sums below zsplit (zsplit N^2)
    double* d_ew[2] = {nullptr, nullptr};
    double edge_rmin = 0, edge_rmax = 0;       // current batch: unpaired pixels' least |m|, any pixel's largest
    double* d_part_sums = nullptr;   // replica partial sums (replicas > 1)
    int* d_status = nullptr;         // device view of h_status (mapped)
    int* h_status = nullptr;         // kernel-reported failures (bounded waits)

    bool timing = false;
    bsg_recon_stats stats{};

    size_t spec_elems() const { return (size_t)(g.ft + 1) * (g.ft + 2); }
    int spec_pitch() const { return g.ft + 2; }
    size_t vol_elems() const { return (size_t)g.map * g.map * g.map; }
};

}  // namespace bsg
