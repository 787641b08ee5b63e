// insert.cu - central-section insertion (fspace_pack_2D +
// fspace_2D_interpolate, bsoft/src/img/Bimage_reconstruct.cpp:25-174).
//
// The reference scatters every pixel q = (h, k) of each padded particle
// transform, q in [-ft/2, ft/2-1]^2, to the map frequency
// m = R (h, k, 0) * inv * mscale and adds F(q) * w to the 1 (nearest) or 8
// (trilinear) voxels around m, with index wrap-around, on a full complex
// N^3 map, plus w to the weight map (and w |F|^2, w^2 to the FOM channels).
//
// Decomposition: one warp owns one tile of the map (8 x 8 x 8, 16 x 16 x 4,
// 16 x 8 x 8 or 16 x 16 x 8 voxels; the autotuner picks the shape) and keeps its
// sums in shared memory in FP32 (each contribution is the float product
// F * w, as the reference forms it), adding them to the FP64 accumulators in
// HBM at the end of the batch.  Nothing else writes the tile, so there are
// no atomics and no block-wide barriers.  The warp tests 32 particles at a
// time against its tile (plane slab and reach, per wrap-around alias) and
// walks the pixels of each particle that reaches it, in particle order.
//
// Conflict-free lanes: the pixels of a particle's footprint are visited on
// a lattice whose points never share a unit cell of the map, one phase
// after another.  Each particle record carries the smallest such lattice
// for its orientation (lattice.h; 5 to 9 phases at step 0.5); without one,
// a lattice safe for every orientation is used (points at least sqrt(3)
// voxels apart: L x L pixels with L = ceil(sqrt(3)/step), step = voxels per
// pixel, or at step 0.5 the 12-phase lattice spanned by (4, 0) and (2, 3)
// pixels).  Two points of a phase have different base voxels floor(m), so
// for any one corner offset the lanes of a warp touch distinct voxels: a
// plain read-modify-write of shared memory is exact.
// The order of every voxel's sum (particle, alias, phase, lattice point,
// corner) is fixed, so results are bitwise reproducible.  Tiles are visited
// heaviest first (nearest to the Fourier origin, where every particle's
// plane passes) so the long ones do not trail the launch, and each tile has
// R replica warps that take consecutive slices of the particle list into
// private partial sums; a combine pass adds the replicas in order.
//
// Each phase's lattice points are enumerated exactly: lane j computes the
// h-interval of lattice row j from the three slab constraints of the tile
// box (once for all phases that walk that row), a warp scan turns the row
// counts into offsets, and lanes take points in order.
#include "context.cuh"

#include <math.h>

namespace bsg {

constexpr int WARPS = 4;                  // warps (tiles) per block

struct InsertArgs {
    const float2* spec;        // batch x (ft+1) x (ft+2), centred
    const DevParticle* part;   // particles of this launch
    int np;
    int half;                  // only particles of this half map (-1: all)
    int N, ft, pitch;
    int ntx, nty, ntz;         // tiles per axis
    const int* order;          // tile visiting order (heaviest first)
    int R;                     // replicas per tile (each takes a slice of the particles)
    double* psum;              // R > 1: replica partial sums, R x channels x N^3
    int zsplit;                // > 0: half-space gridding (walk_edges)
    double2* evol;             // half-space: unpaired pixels' sums below zsplit (zsplit x N^2)
    double* ew;
    double edge_rmin;          // unpaired pixels lie at least this far from the origin (voxels)
    double edge_rmax;          // and no pixel farther than this
    int interp;
    double maxs2, mins2, mscale;
    double2* vol;
    double* w;
    double* pow;
    double* w2;
};

// Does particle P's plane come within reach of the tile for alias
// combination a (bit i set: axis i shifted by -N)?  Bitmask over the 8.
template <int TX, int TY, int TZ>
__device__ __forceinline__ unsigned tile_mask(const DevParticle& P, int x0, int y0, int z0, int N, int ft) {
    unsigned mask = 0;
    const float ex = 0.5f * (TX - 1), ey = 0.5f * (TY - 1), ez = 0.5f * (TZ - 1);
    const float hf = 0.5f * ft;
    // (an Ewald surface deviates from the plane by up to P.ezmax voxels)
    const float rx = hf * (fabsf(P.af[0]) + fabsf(P.bf[0])) + 1.0f + P.ezmax;
    const float ry = hf * (fabsf(P.af[1]) + fabsf(P.bf[1])) + 1.0f + P.ezmax;
    const float rz = hf * (fabsf(P.af[2]) + fabsf(P.bf[2])) + 1.0f + P.ezmax;
    const float n0 = (float)P.nrm[0], n1 = (float)P.nrm[1], n2 = (float)P.nrm[2];
    const float slack = P.slab + fabsf(n0) * ex + fabsf(n1) * ey + fabsf(n2) * ez + 1e-3f + P.ezmax;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const float cx = x0 - ((a & 1) ? N : 0) + ex;
        const float cy = y0 - ((a & 2) ? N : 0) + ey;
        const float cz = z0 - ((a & 4) ? N : 0) + ez;
        if (fabsf(cx) - ex > rx || fabsf(cy) - ey > ry || fabsf(cz) - ez > rz) continue;
        if (fabsf(n0 * cx + n1 * cy + n2 * cz) > slack) continue;
        mask |= 1u << a;
    }
    return mask;
}

__device__ __forceinline__ float pixel_weight_gate(const InsertArgs& a, const DevParticle& P, int h, int k,
                                                   bool& keep) {
    // s2 as fspace_pack_2D forms it: s = (h, k) * inv in double
    const double inv = sqrt(P.inv2);
    const double sx = h * inv, sy = k * inv;
    const double s2 = sx * sx + sy * sy;
    keep = (s2 >= a.mins2 && s2 <= a.maxs2);
    const double d = (a.maxs2 - s2) * a.mscale;
    return d < 1.0 ? (float)sqrt(d > 0 ? d : 0.0) : 1.0f;
}

// Tile sums are FP32: one batch adds at most a few thousand contributions
// to a voxel, each the float product F * w the reference forms; the batch's
// sums are folded into the FP64 map accumulators, which carry the long
// reduction over all particles.
typedef float tacc_t;

struct TileAcc {
    tacc_t* re;
    tacc_t* im;
    tacc_t* w;
    tacc_t* p;
    tacc_t* q;
};

template <bool FOM>
__device__ __forceinline__ void add_voxel(const TileAcc& A, int i, float2 f, float w) {
    A.re[i] += f.x * w;
    A.im[i] += f.y * w;
    A.w[i] += w;
    if (FOM) {
        A.p[i] += w * (f.x * f.x + f.y * f.y);
        A.q[i] += w * w;
    }
}

// One pixel (h, k) of particle P against the tile at alias origin o.  All
// lanes of the warp call this together (`act` false for idle lanes); the
// __syncwarp after each corner orders the shared-memory updates of
// different corner offsets, which may touch the same voxel from different
// lanes.
template <bool FOM, bool GATE, int TX, int TY, int TZ>
__device__ __forceinline__ void pixel(const InsertArgs& a, const DevParticle& P, const float2* S, const TileAcc& A,
                                      double ox, double oy, double oz, int h, int k, bool act) {
    const int hf = a.ft / 2;
    float wt = P.pw;
    if (GATE && act) {
        bool keep;
        const float tw = pixel_weight_gate(a, P, h, k, keep);
        if (!keep) act = false;
        wt *= tw;
    }
    // map frequency relative to the tile origin, in double as the reference
    // forms it
    double mx = h * P.ad[0] + k * P.bd[0] - ox;
    double my = h * P.ad[1] + k * P.bd[1] - oy;
    double mz = h * P.ad[2] + k * P.bd[2] - oz;
    if (P.ewh != 0.0) {
        // Ewald surface: s_z = +-(lambda/2) s2 along R[:,2] (Bimage_reconstruct.cpp:157-168)
        const double sx = h * P.inv, sy = k * P.inv, sz = P.ewh * (sx * sx + sy * sy);
        mx += sz * P.cd[0];
        my += sz * P.cd[1];
        mz += sz * P.cd[2];
    }
    const float2 f = act ? __ldg(S + (size_t)(k + hf) * a.pitch + (h + hf)) : make_float2(0.f, 0.f);
    if (a.interp != 2) {
        const double fx = floor(mx + 0.5), fy = floor(my + 0.5), fz = floor(mz + 0.5);
        const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
        float w = wt;
        if (a.interp == 1) {
            const double dx = mx - fx, dy = my - fy, dz = mz - fz;
            w = (float)((double)wt * (1.0 - sqrt(dx * dx + dy * dy + dz * dz)));
        }
        if (act && (unsigned)ix < TX && (unsigned)iy < TY && (unsigned)iz < TZ && w > 0.f)
            add_voxel<FOM>(A, (iz * TY + iy) * TX + ix, f, w);
        __syncwarp();
        return;
    }
    const double flx = floor(mx), fly = floor(my), flz = floor(mz);
    const int ix = (int)flx, iy = (int)fly, iz = (int)flz;
    const float rx = (float)(mx - flx), ry = (float)(my - fly), rz = (float)(mz - flz);
#pragma unroll
    for (int dz = 0; dz < 2; ++dz) {
        const int z = iz + dz;
        const float wz = dz ? rz : 1.f - rz;
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
            const int y = iy + dy;
            const float wyz = (dy ? ry : 1.f - ry) * wz * wt;
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int x = ix + dx;
                if (act && (unsigned)x < TX && (unsigned)y < TY && (unsigned)z < TZ)
                    add_voxel<FOM>(A, (z * TY + y) * TX + x, f, (dx ? rx : 1.f - rx) * wyz);
                __syncwarp();
            }
        }
    }
}

// Walk the pixels of particle P (alias origin o) whose contributions can
// reach the tile, phase by phase of the lattice, calling pix(h, k, act) with
// all lanes of the warp together (act false for idle lanes).
template <int TX, int TY, int TZ, class Pix>
__device__ __forceinline__ void walk_pair(const DevParticle& P, int hf, double ox, double oy, double oz, int lane,
                                          int* s_row, Pix&& pix) {
    // open box of map frequencies whose tent touches the tile (an Ewald
    // surface adds up to P.ezmax voxels to every coordinate)
    const double e = P.ezmax;
    const double lo[3] = {ox - 1.0 - e, oy - 1.0 - e, oz - 1.0 - e};
    const double hi[3] = {ox + TX + e, oy + TY + e, oz + TZ + e};
    double vc = 0, hv = 0, uc = 0, hu = 0;
    for (int i = 0; i < 3; ++i) {
        const double c = 0.5 * (lo[i] + hi[i]), e = 0.5 * (hi[i] - lo[i]);
        vc += P.bd[i] * c; hv += fabs(P.bd[i]) * e;
        uc += P.ad[i] * c; hu += fabs(P.ad[i]) * e;
    }
    vc *= P.inv_st2; hv *= P.inv_st2; uc *= P.inv_st2; hu *= P.inv_st2;
    const int k_lo = max((int)ceil(vc - hv), -hf), k_hi = min((int)floor(vc + hv), hf - 1);
    const int h_lo = max((int)ceil(uc - hu), -hf), h_hi = min((int)floor(uc + hu), hf - 1);
    if (k_lo > k_hi || h_lo > h_hi) return;
    // Conflict-free lattice: two points of one phase never share a unit cell
    // of the map.  P.lat, when set, is the smallest such lattice for this
    // particle's orientation (lattice.h; 5 to 9 phases at step 0.5).  Else
    // one safe for every orientation, whose points are >= sqrt(3) voxels
    // apart: the square lattice of L x L pixels (L = ceil(sqrt(3)/step)), or,
    // where it has fewer phases, the lattice spanned by (4, 0) and (2, 3)
    // pixels (shortest vector sqrt(13) pixels; 12 phases at step 0.5).
    // Row j of phase (ph, pk) is k = k_lo + pk + Lk j, its points
    // h = h_lo + ph + sh j + Lh i.
    int Lh, Lk, sh;
    if (P.lat) {
        Lh = P.lat & 0xfff; Lk = (P.lat >> 12) & 0xfff; sh = (P.lat >> 24) & 0x7f;
    } else {
        const int L = max(1, (int)ceilf(1.7320508f * 1.0001f * P.inv_step));
        if (L * L > 12 && 3.6055513f * P.step >= 1.7320508f * 1.0001f) { Lh = 4; Lk = 3; sh = 2; }
        else { Lh = L; Lk = L; sh = 0; }
    }
    // per-axis 1 / ad (0 when the axis does not vary along h)
    const double* ia = P.iad;
    for (int pk = 0; pk < Lk; ++pk) {
        const int k0 = k_lo + pk;
        if (k0 > k_hi) break;
        const int nrows = (k_hi - k0) / Lk + 1;
        for (int jb = 0; jb < nrows; jb += 32) {
            // lane j: the exact h range [hl, hh] of row k = k0 + Lk (jb + j),
            // shared by the Lh phases that walk this row
            const int j = jb + lane;
            const int k = k0 + Lk * j;
            double hl = h_lo, hh = h_hi;
            bool live = j < nrows;
            if (live) {
                for (int i = 0; i < 3; ++i) {
                    const double base = k * P.bd[i];
                    if (ia[i] != 0.0) {
                        double p0 = (lo[i] - base) * ia[i], p1 = (hi[i] - base) * ia[i];
                        if (p0 > p1) { const double t = p0; p0 = p1; p1 = t; }
                        hl = fmax(hl, p0);
                        hh = fmin(hh, p1);
                    } else if (!(base > lo[i] && base < hi[i])) {
                        live = false;
                    }
                }
                live = live && hl <= hh;
            }
            for (int ph = 0; ph < Lh; ++ph) {
                if (sh == 0 && h_lo + ph > h_hi) break;
                int hfirst = 0, cnt = 0;
                if (live) {
                    // lattice h = h0 + Lh i inside [hl, hh]
                    const int h0 = h_lo + ph + sh * j;
                    const int i0 = (int)ceil((hl - h0) / Lh), i1 = (int)floor((hh - h0) / Lh);
                    if (i1 >= i0) { hfirst = h0 + Lh * i0; cnt = i1 - i0 + 1; }
                }
                // exclusive scan of the row counts
                int incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                const int total = __shfl_sync(0xffffffffu, incl, 31);
                if (total == 0) continue;
                s_row[lane] = incl;                        // inclusive end of row j
                s_row[32 + lane] = hfirst;
                s_row[64 + lane] = k;
                __syncwarp();
                for (int t0 = 0; t0 < total; t0 += 32) {
                    const int t = t0 + lane;
                    const bool act = t < total;
                    int r = 0;                              // row holding point t
#pragma unroll
                    for (int sft = 16; sft > 0; sft >>= 1)
                        if (s_row[r + sft - 1] <= t) r += sft;
                    r = min(r, 31);
                    const int before = r ? s_row[r - 1] : 0;
                    const int h = s_row[32 + r] + Lh * (t - before);
                    pix(h, s_row[64 + r], act);
                }
                __syncwarp();
            }
        }
    }
}

// floor(x / d) for 0 < d and |x| < 2^20, from an approximate reciprocal of
// d: the float quotient is within one of the answer, and the remainder
// corrects it (the integers a division would give, without one per row).
__device__ __forceinline__ int floor_div(int x, int d, float inv_d) {
    int q = __float2int_rd((float)x * inv_d);
    int r = x - q * d;
    if (r < 0) { --q; r += d; }
    if (r >= d) ++q;
    return q;
}

// The same walk with the lattice phases of one row block interleaved: lane t
// takes a group of Lh consecutive pixels of one lattice row (h = g, g + 1,
// ..., g + Lh - 1 with g = h_lo + sh j + Lh i), one pixel of each column
// phase, and the warp steps through the phases together: at step ph every
// lane holds a point of phase (ph, pk), so the conflict-free property of a
// phase still holds, and pix() ends each step with __syncwarp.  The row
// search is done once per group instead of once per point, and neighbouring
// lanes read neighbouring pixels of the spectrum.
// excl = 1 leaves out the row k = -hf and the column h = -hf (half-space
// gridding grids them separately, walk_edges).
template <int TX, int TY, int TZ, class Pix>
__device__ __forceinline__ void walk_groups(const DevParticle& P, int hf, double ox, double oy, double oz, int lane,
                                            int* s_row, int excl, Pix&& pix) {
    const double e = P.ezmax;
    const double lo[3] = {ox - 1.0 - e, oy - 1.0 - e, oz - 1.0 - e};
    const double hi[3] = {ox + TX + e, oy + TY + e, oz + TZ + e};
    double vc = 0, hv = 0, uc = 0, hu = 0;
    for (int i = 0; i < 3; ++i) {
        const double c = 0.5 * (lo[i] + hi[i]), e = 0.5 * (hi[i] - lo[i]);
        vc += P.bd[i] * c; hv += fabs(P.bd[i]) * e;
        uc += P.ad[i] * c; hu += fabs(P.ad[i]) * e;
    }
    vc *= P.inv_st2; hv *= P.inv_st2; uc *= P.inv_st2; hu *= P.inv_st2;
    const int k_lo = max((int)ceil(vc - hv), -hf + excl), k_hi = min((int)floor(vc + hv), hf - 1);
    const int h_lo = max((int)ceil(uc - hu), -hf + excl), h_hi = min((int)floor(uc + hu), hf - 1);
    if (k_lo > k_hi || h_lo > h_hi) return;
    int Lh, Lk, sh;
    if (P.lat) {
        Lh = P.lat & 0xfff; Lk = (P.lat >> 12) & 0xfff; sh = (P.lat >> 24) & 0x7f;
    } else {
        const int L = max(1, (int)ceilf(1.7320508f * 1.0001f * P.inv_step));
        if (L * L > 12 && 3.6055513f * P.step >= 1.7320508f * 1.0001f) { Lh = 4; Lk = 3; sh = 2; }
        else { Lh = L; Lk = L; sh = 0; }
    }
    const double* ia = P.iad;
    const float iLh = __fdividef(1.0f, (float)Lh);
    for (int pk = 0; pk < Lk; ++pk) {
        const int k0 = k_lo + pk;
        if (k0 > k_hi) break;
        for (int jb = 0; k0 + Lk * jb <= k_hi; jb += 32) {
            const int j = jb + lane;
            const int k = k0 + Lk * j;
            double hl = h_lo, hh = h_hi;
            bool live = k <= k_hi;
            if (live) {
                for (int i = 0; i < 3; ++i) {
                    const double base = k * P.bd[i];
                    if (ia[i] != 0.0) {
                        double p0 = (lo[i] - base) * ia[i], p1 = (hi[i] - base) * ia[i];
                        if (p0 > p1) { const double t = p0; p0 = p1; p1 = t; }
                        hl = fmax(hl, p0);
                        hh = fmin(hh, p1);
                    } else if (!(base > lo[i] && base < hi[i])) {
                        live = false;
                    }
                }
                live = live && hl <= hh;
            }
            // this row's pixels [hmin, hmax] in groups of Lh from its phase-0
            // lattice point g0 = h_lo + sh j (mod Lh)
            int gfirst = 0, cnt = 0, hmin = 0, hmax = -1;
            if (live) {
                hmin = (int)ceil(hl);
                hmax = (int)floor(hh);
                if (hmax >= hmin) {
                    const int g0 = h_lo + sh * j;
                    const int i0 = floor_div(hmin - g0, Lh, iLh);
                    const int i1 = floor_div(hmax - g0, Lh, iLh);
                    gfirst = g0 + Lh * i0;
                    cnt = i1 - i0 + 1;
                }
            }
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            if (total == 0) continue;
            s_row[lane] = incl;                        // inclusive end of row j's groups
            s_row[32 + lane] = gfirst;
            s_row[64 + lane] = k;
            s_row[96 + lane] = hmin;
            s_row[128 + lane] = hmax;
            __syncwarp();
            for (int t0 = 0; t0 < total; t0 += 32) {
                const int t = t0 + lane;
                const bool in = t < total;
                int r = 0;                              // row holding group t
#pragma unroll
                for (int sft = 16; sft > 0; sft >>= 1)
                    if (s_row[r + sft - 1] <= t) r += sft;
                r = min(r, 31);
                const int before = r ? s_row[r - 1] : 0;
                const int g = s_row[32 + r] + Lh * (t - before);
                const int kr = s_row[64 + r], lo_h = s_row[96 + r], hi_h = s_row[128 + r];
                for (int ph = 0; ph < Lh; ++ph) {
                    const int h = g + ph;
                    pix(h, kr, in && h >= lo_h && h <= hi_h);
                }
            }
            __syncwarp();
        }
    }
}

// Half-space gridding.  A real image's transform is Hermitian, F(-q) =
// conj(F(q)), and a pixel q and its mate -q land at mirrored map positions
// m and -m (m is linear in q) with mirrored trilinear corners of equal
// weights.  So the sums P of the pixels that have their mate in the stored
// transform (q in [-ft/2, ft/2 - 1]^2) satisfy P(-v) = conj(P(v)),
// P_w(-v) = P_w(v); the others - the row k = -ft/2 and the column
// h = -ft/2 - make sums U of their own.  With zsplit > N/2 (so every voxel
// or its mirror lies below it), the tiles below zsplit grid P (walk_groups
// without the unpaired pixels) into the map accumulators and U into evol /
// ew; the tiles at or above zsplit grid only U, into the map accumulators.
// Reading the map gives P(v) + U(v) below the split and conj(P(-v)) + U(v)
// above it: sums of the same contributions as the full map's, none of them
// subtracted, so a voxel that nothing reaches reads exactly zero.
// walk_edges visits the unpaired pixels whose tents reach the tile, one
// line at a time, points L pixels apart (L step >= sqrt(3) voxels) so that
// the lanes of a call touch distinct cells; pix(h, k, act) as walk_groups.
template <int TX, int TY, int TZ, class Pix>
__device__ __forceinline__ void walk_edges(const DevParticle& P, int hf, double ox, double oy, double oz, int lane,
                                           Pix&& pix) {
    const double lo[3] = {ox - 1.0, oy - 1.0, oz - 1.0};
    const double hi[3] = {ox + TX, oy + TY, oz + TZ};
    const int L = max(1, (int)ceilf(1.7320508f * 1.0001f * P.inv_step));
    for (int line = 0; line < 2; ++line) {
        // 0: (t, -hf), t in [-hf, hf - 1];  1: (-hf, t), t in [-hf + 1, hf - 1]
        const bool along_h = line == 0;
        double tl = line == 0 ? -hf : -hf + 1;
        double th = hf - 1;
        bool live = true;
        for (int i = 0; i < 3; ++i) {
            const double idir = along_h ? P.iad[i] : P.ibd[i];
            const double base = -hf * (along_h ? P.bd[i] : P.ad[i]);
            if (idir != 0.0) {
                double p0 = (lo[i] - base) * idir, p1 = (hi[i] - base) * idir;
                if (p0 > p1) { const double t = p0; p0 = p1; p1 = t; }
                tl = fmax(tl, p0);
                th = fmin(th, p1);
            } else if (!(base >= lo[i] && base <= hi[i])) {
                live = false;
            }
        }
        if (!live) continue;
        const int t0 = (int)ceil(tl), t1 = (int)floor(th);
        for (int ph = 0; ph < L; ++ph) {
            const int first = t0 + ph;
            if (first > t1) break;
            for (int tb = first; tb <= t1; tb += 32 * L) {
                const int t = tb + L * lane;
                pix(along_h ? t : -hf, along_h ? -hf : t, t <= t1);
            }
        }
    }
}

// Can an unpaired pixel (at least rmin voxels from the origin, and no pixel
// beyond rmax) reach the tile, under some wrap-around alias?
template <int TX, int TY, int TZ>
__device__ __forceinline__ bool tile_reaches_edges(int x0, int y0, int z0, int N, double rmin, double rmax) {
    const int o[3] = {x0, y0, z0}, T[3] = {TX, TY, TZ};
    for (int a = 0; a < 8; ++a) {
        double nr = 0, fr = 0;
        for (int i = 0; i < 3; ++i) {
            const double lo = o[i] - (((a >> i) & 1) ? N : 0) - 1.0, hi = lo + T[i] + 1.0;
            const double n = (lo <= 0 && hi >= 0) ? 0.0 : fmin(fabs(lo), fabs(hi));
            const double f = fmax(fabs(lo), fabs(hi));
            nr += n * n;
            fr += f * f;
        }
        if (nr <= rmax * rmax && fr >= rmin * rmin) return true;
    }
    return false;
}

template <bool FOM, bool GATE, int TX, int TY, int TZ>
__device__ __forceinline__ void scatter_particle(const InsertArgs& a, const DevParticle& P, const float2* S,
                                                 const TileAcc& A, double ox, double oy, double oz, int lane,
                                                 int* s_row) {
    walk_pair<TX, TY, TZ>(P, a.ft / 2, ox, oy, oz, lane, s_row, [&](int h, int k, bool act) {
        pixel<FOM, GATE, TX, TY, TZ>(a, P, S, A, ox, oy, oz, h, k, act);
    });
}

// Tile sums -> HBM: added to the map accumulators (one replica), or stored
// into this replica's partial buffer (combined later in replica order).
template <bool FOM, int TX, int TY, int TZ>
__device__ __forceinline__ void fold_tile(const InsertArgs& a, const TileAcc& A, int x0, int y0, int z0, int r,
                                          int lane) {
    const int N = a.N;
    constexpr int TV = TX * TY * TZ;
    const size_t N3 = (size_t)N * N * N;
    const int nch = FOM ? 5 : 3;
    for (int i = lane; i < TV; i += 32) {
        const int lx = i % TX, ly = (i / TX) % TY, lz = i / (TX * TY);
        const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
        if (x < N && y < N && z < N) {
            const size_t idx = ((size_t)z * N + y) * N + x;
            if (a.R > 1) {
                double* pb = a.psum + (size_t)r * nch * N3 + idx;
                pb[0] = A.re[i];
                pb[N3] = A.im[i];
                pb[2 * N3] = A.w[i];
                if (FOM) { pb[3 * N3] = A.p[i]; pb[4 * N3] = A.q[i]; }
            } else {
                double2 o = a.vol[idx];
                o.x += A.re[i];
                o.y += A.im[i];
                a.vol[idx] = o;
                a.w[idx] += A.w[i];
                if (FOM) { a.pow[idx] += A.p[i]; a.w2[idx] += A.q[i]; }
            }
        }
        A.re[i] = 0; A.im[i] = 0; A.w[i] = 0;
        if (FOM) { A.p[i] = 0; A.q[i] = 0; }
    }
    __syncwarp();
}

template <bool FOM, bool GATE, int TX, int TY, int TZ>
__global__ void __launch_bounds__(WARPS * 32) insert_kernel(InsertArgs a) {
    constexpr int NCH = FOM ? 5 : 3;
    constexpr int TV = TX * TY * TZ;
    extern __shared__ tacc_t s_dacc[];                 // WARPS x NCH x TV
    tacc_t* const my_acc = s_dacc + (size_t)(threadIdx.x >> 5) * NCH * TV;
    __shared__ int s_rows[WARPS][96];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gw = blockIdx.x * WARPS + warp;
    const int slot = gw / a.R, rep = gw % a.R;       // replicas of a tile are adjacent
    if (slot >= a.ntx * a.nty * a.ntz) return;
    const int tile = a.order[slot];
    // this replica's slice of the particles
    const int p_lo = (int)((long)a.np * rep / a.R), p_hi = (int)((long)a.np * (rep + 1) / a.R);
    const int x0 = (tile % a.ntx) * TX, y0 = ((tile / a.ntx) % a.nty) * TY, z0 = (tile / (a.ntx * a.nty)) * TZ;
    const int N = a.N;
    const int hf = a.ft / 2;
    const size_t spec_stride = (size_t)(2 * hf + 1) * a.pitch;
    TileAcc A;
    A.re = my_acc; A.im = A.re + TV; A.w = A.im + TV;
    A.p = FOM ? A.w + TV : nullptr; A.q = FOM ? A.p + TV : nullptr;
    for (int i = lane; i < NCH * TV; i += 32) my_acc[i] = 0;
    __syncwarp();

    for (int base = p_lo; base < p_hi; base += 32) {
        const int p = base + lane;
        unsigned mask = 0;
        if (p < p_hi) {
            const DevParticle& P = a.part[p];
            if (P.half == a.half || a.half < 0) mask = tile_mask<TX, TY, TZ>(P, x0, y0, z0, N, a.ft);
        }
        unsigned todo = __ballot_sync(0xffffffffu, mask != 0);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const unsigned am = __shfl_sync(0xffffffffu, mask, src);
            const int pi = base + src;
            const DevParticle& P = a.part[pi];
            const float2* S = a.spec + (size_t)P.spec * spec_stride;
            for (int al = 0; al < 8; ++al)
                if ((am >> al) & 1u)
                    scatter_particle<FOM, GATE, TX, TY, TZ>(a, P, S, A, (double)(x0 - ((al & 1) ? N : 0)),
                                                (double)(y0 - ((al & 2) ? N : 0)),
                                                (double)(z0 - ((al & 4) ? N : 0)), lane, s_rows[warp]);
        }
    }
    fold_tile<FOM, TX, TY, TZ>(a, A, x0, y0, z0, rep, lane);
}

// ---- gridding without the FOM channels: float4 cells --------------------
//
// The map tile is an array of float4 cells {F re * w, F im * w, w, unused},
// so a corner's read-modify-write is one 16-byte load, three adds and one
// 16-byte store.  Cell (x, y, z) of the tile sits at slot x + PX y + PP z:
// the plane pitch PP (PX TY plus a few unused slots) spreads the cells a
// warp's lattice points touch over the eight 16-byte bank groups (at 8^3,
// PP = 68 puts cell (x, y, z) in group (x + 4 z) mod 8; the pitches were
// chosen by simulating the lattice walk over random orientations), and the
// corner offsets stay compile-time constants.
//
// Map frequencies are formed in FP32 relative to the tile: per (tile,
// particle) pair an anchor pixel (hc, kc) near the tile's projection has its
// frequency hc ad + kc bd - o formed in FP64, and a point (h, k) adds
// (h - hc) af + (k - kc) bf to it.  The offsets are at most ~25 pixel steps
// at these tile sizes, so the coordinates carry < 5e-6 voxel of rounding;
// the trilinear weights are continuous in the coordinates, so a floor that
// lands on the other side of a cell boundary because of it moves a
// contribution by that much, and the phase lattices keep a margin above it
// (lattice.h).
// One cell's read-modify-write as a single 16-byte shared load and store
// (the unused fourth word travels with them, so the compiler cannot split the
// access into narrower ones).
__device__ __forceinline__ void cell_add(unsigned addr, float2 f, float w) {
    float x, y, z, u;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(x), "=f"(y), "=f"(z), "=f"(u) : "r"(addr) : "memory");
    x = fmaf(f.x, w, x);
    y = fmaf(f.y, w, y);
    z += w;
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" :: "r"(addr), "f"(x), "f"(y), "f"(z), "f"(u) : "memory");
}

template <bool GATE, bool EW, int TX, int TY, int TZ, int PX, int PP>
__device__ __forceinline__ void pixel4(const InsertArgs& a, const DevParticle& P, const float2* S, float4* cell,
                                       unsigned cell0,
                                       float bx, float by, float bz, int hc, int kc, int h, int k, bool act) {
    const int hf = a.ft / 2;
    float wt = P.pw;
    if (GATE && act) {
        bool keep;
        const float tw = pixel_weight_gate(a, P, h, k, keep);
        if (!keep) act = false;
        wt *= tw;
    }
    const float dh = (float)(h - hc), dk = (float)(k - kc);
    float mx = fmaf(dh, P.af[0], fmaf(dk, P.bf[0], bx));
    float my = fmaf(dh, P.af[1], fmaf(dk, P.bf[1], by));
    float mz = fmaf(dh, P.af[2], fmaf(dk, P.bf[2], bz));
    if (EW && P.ewh != 0.0) {
        // Ewald surface: s_z = +-(lambda/2) s2 along R[:,2] (Bimage_reconstruct.cpp:
        // 157-168), at most P.ezmax voxels, added in FP32 to the tile-relative
        // coordinate (the lattice keeps a margin for its variation)
        const double sx = h * P.inv, sy = k * P.inv, sz = P.ewh * (sx * sx + sy * sy);
        mx += (float)(sz * P.cd[0]);
        my += (float)(sz * P.cd[1]);
        mz += (float)(sz * P.cd[2]);
    }
    const float2 f = act ? __ldg(S + (size_t)(k + hf) * a.pitch + (h + hf)) : make_float2(0.f, 0.f);
    if (a.interp != 2) {
        const float fx = floorf(mx + 0.5f), fy = floorf(my + 0.5f), fz = floorf(mz + 0.5f);
        const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
        float w = wt;
        if (a.interp == 1) {
            const float dx = mx - fx, dy = my - fy, dz = mz - fz;
            w = wt * (1.0f - sqrtf(dx * dx + dy * dy + dz * dz));
        }
        if (act && (unsigned)ix < TX && (unsigned)iy < TY && (unsigned)iz < TZ && w > 0.f)
            cell_add(cell0 + 16u * (unsigned)(ix + PX * iy + PP * iz), f, w);
        __syncwarp();
        return;
    }
    const float flx = floorf(mx), fly = floorf(my), flz = floorf(mz);
    const int ix = (int)flx, iy = (int)fly, iz = (int)flz;
    const float rx = mx - flx, ry = my - fly, rz = mz - flz;
    const bool vx[2] = {(unsigned)ix < TX, (unsigned)(ix + 1) < TX};
    const bool vy[2] = {(unsigned)iy < TY, (unsigned)(iy + 1) < TY};
    const bool vz[2] = {(unsigned)iz < TZ, (unsigned)(iz + 1) < TZ};
    const unsigned cell_addr = cell0 + 16u * (unsigned)(ix + PX * iy + PP * iz);
#pragma unroll
    for (int dz = 0; dz < 2; ++dz) {
        const float wz = (dz ? rz : 1.f - rz) * wt;
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
            const float wyz = (dy ? ry : 1.f - ry) * wz;
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                if (act && vx[dx] && vy[dy] && vz[dz]) {
                    const float w = (dx ? rx : 1.f - rx) * wyz;
                    cell_add(cell_addr + 16u * (unsigned)(dx + PX * dy + PP * dz), f, w);
                }
                __syncwarp();
            }
        }
    }
}

template <bool GATE, bool EW, int TX, int TY, int TZ, int PX, int PP, int NW>
__global__ void __launch_bounds__(NW * 32, 5) grid4_kernel(InsertArgs a) {
    constexpr int SLOTS = PP * TZ;
    constexpr int TV = TX * TY * TZ;
    extern __shared__ float4 s_cells[];                 // NW x SLOTS
    __shared__ int s_rows[NW][160];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float4* const cell = s_cells + (size_t)warp * SLOTS;
    const int gw = blockIdx.x * NW + warp;
    const int slot = gw / a.R, rep = gw % a.R;        // replicas of a tile are adjacent
    if (slot >= a.ntx * a.nty * a.ntz) return;
    const int tile = a.order[slot];
    const int p_lo = (int)((long)a.np * rep / a.R), p_hi = (int)((long)a.np * (rep + 1) / a.R);
    const int x0 = (tile % a.ntx) * TX, y0 = ((tile / a.ntx) % a.nty) * TY, z0 = (tile / (a.ntx * a.nty)) * TZ;
    const int N = a.N;
    const int hf = a.ft / 2;
    const size_t spec_stride = (size_t)(2 * hf + 1) * a.pitch;
    const unsigned cell0 = (unsigned)__cvta_generic_to_shared(cell);
    // half-space gridding (walk_edges): tiles at or above zsplit grid only
    // the unpaired pixels; those below it grid the others, and then (one
    // replica, all particles) the unpaired ones into evol / ew
    const bool hs = a.zsplit > 0;
    const bool upper = hs && z0 >= a.zsplit;
    const bool edges = hs && tile_reaches_edges<TX, TY, TZ>(x0, y0, z0, N, a.edge_rmin, a.edge_rmax);
    for (int i = lane; i < SLOTS; i += 32) cell[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncwarp();

    // pass 0: the tile's sums (all pixels; with half-space gridding the
    // paired ones, or above the split the unpaired ones); pass 1: the
    // unpaired pixels of a tile below the split
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1 && !(hs && !upper && edges && rep == 0)) break;
        const bool edge_walk = pass == 1 || upper;
        const int b_lo = pass ? 0 : p_lo, b_hi = pass ? a.np : p_hi;
        // (a tile that no unpaired pixel reaches skips the edge walks)
        const int b_end = (edge_walk && !edges) ? b_lo : b_hi;
        for (int base = b_lo; base < b_end; base += 32) {
            const int p = base + lane;
            unsigned mask = 0;
            if (p < b_hi) {
                const DevParticle& P = a.part[p];
                if (P.half == a.half || a.half < 0) mask = tile_mask<TX, TY, TZ>(P, x0, y0, z0, N, a.ft);
            }
            unsigned todo = __ballot_sync(0xffffffffu, mask != 0);
            while (todo) {
                const int src = __ffs(todo) - 1;
                todo &= todo - 1;
                const unsigned am = __shfl_sync(0xffffffffu, mask, src);
                const DevParticle& P = a.part[base + src];
                const float2* S = a.spec + (size_t)P.spec * spec_stride;
                for (int al = 0; al < 8; ++al) {
                    if (!((am >> al) & 1u)) continue;
                    const double ox = (double)(x0 - ((al & 1) ? N : 0));
                    const double oy = (double)(y0 - ((al & 2) ? N : 0));
                    const double oz = (double)(z0 - ((al & 4) ? N : 0));
                    // anchor pixel: the tile centre's projection on the plane
                    const double cx = ox + 0.5 * (TX - 1), cy = oy + 0.5 * (TY - 1), cz = oz + 0.5 * (TZ - 1);
                    const int hc = (int)rint((P.ad[0] * cx + P.ad[1] * cy + P.ad[2] * cz) * P.inv_st2);
                    const int kc = (int)rint((P.bd[0] * cx + P.bd[1] * cy + P.bd[2] * cz) * P.inv_st2);
                    const float bx = (float)(hc * P.ad[0] + kc * P.bd[0] - ox);
                    const float by = (float)(hc * P.ad[1] + kc * P.bd[1] - oy);
                    const float bz = (float)(hc * P.ad[2] + kc * P.bd[2] - oz);
                    auto pix = [&](int h, int k, bool act) {
                        pixel4<GATE, EW, TX, TY, TZ, PX, PP>(a, P, S, cell, cell0, bx, by, bz, hc, kc, h, k, act);
                    };
                    if (edge_walk) walk_edges<TX, TY, TZ>(P, hf, ox, oy, oz, lane, pix);
                    else walk_groups<TX, TY, TZ>(P, hf, ox, oy, oz, lane, s_rows[warp], hs ? 1 : 0, pix);
                }
            }
        }
        // tile sums -> HBM: pass 0 adds to the map (one replica) or stores
        // this replica's partial sums (combined later in replica order);
        // pass 1 adds to evol / ew.  The cells are cleared for the next pass.
        const size_t N3 = (size_t)N * N * N;
        for (int i = lane; i < TV; i += 32) {
            const int lx = i % TX, ly = (i / TX) % TY, lz = i / (TX * TY);
            const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
            const int ci = lx + PX * ly + PP * lz;
            const float4 c = cell[ci];
            if (x < N && y < N && z < N) {
                const size_t idx = ((size_t)z * N + y) * N + x;
                if (pass == 1) {
                    double2 o = a.evol[idx];
                    o.x += c.x;
                    o.y += c.y;
                    a.evol[idx] = o;
                    a.ew[idx] += c.z;
                } else if (a.R > 1) {
                    double* pb = a.psum + (size_t)rep * 3 * N3 + idx;
                    pb[0] = c.x;
                    pb[N3] = c.y;
                    pb[2 * N3] = c.z;
                } else {
                    double2 o = a.vol[idx];
                    o.x += c.x;
                    o.y += c.y;
                    a.vol[idx] = o;
                    a.w[idx] += c.z;
                }
            }
            cell[ci] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncwarp();
    }
}

// vol += sum over replicas, in replica order.
template <bool FOM>
__global__ void combine_kernel(InsertArgs a) {
    const size_t N3 = (size_t)a.N * a.N * a.N;
    const int nch = FOM ? 5 : 3;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N3; i += (size_t)gridDim.x * blockDim.x) {
        double re = 0, im = 0, w = 0, p = 0, q = 0;
        for (int r = 0; r < a.R; ++r) {
            const double* pb = a.psum + (size_t)r * nch * N3 + i;
            re += pb[0]; im += pb[N3]; w += pb[2 * N3];
            if (FOM) { p += pb[3 * N3]; q += pb[4 * N3]; }
        }
        double2 o = a.vol[i];
        o.x += re; o.y += im;
        a.vol[i] = o;
        a.w[i] += w;
        if (FOM) { a.pow[i] += p; a.w2[i] += q; }
    }
}

// Tile shapes the autotuner chooses from (map voxels per warp).  The float4
// cell pitches (PX, PP) and warps per block of each shape are the template
// arguments of its grid4_kernel launch below.
struct Shape { int tx, ty, tz; };
static const Shape kShapes[] = {{8, 8, 8}, {16, 16, 4}, {16, 8, 8}, {16, 16, 8}};
constexpr int kNumShapes = 4;

int insert_num_shapes() { return kNumShapes; }
void insert_shape(int i, int* tx, int* ty, int* tz) { *tx = kShapes[i].tx; *ty = kShapes[i].ty; *tz = kShapes[i].tz; }

template <int TX, int TY, int TZ>
static cudaError_t set_smem_shape() {
    const int smem = (int)(WARPS * 5 * TX * TY * TZ * sizeof(tacc_t));
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(insert_kernel<true, true, TX, TY, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(insert_kernel<true, false, TX, TY, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(insert_kernel<false, true, TX, TY, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(insert_kernel<false, false, TX, TY, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

template <int TX, int TY, int TZ, int PX, int PP, int NW>
static cudaError_t set_smem_shape4() {
    const int smem = (int)(NW * PP * TZ * sizeof(float4));
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(grid4_kernel<true, false, TX, TY, TZ, PX, PP, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(grid4_kernel<false, false, TX, TY, TZ, PX, PP, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(grid4_kernel<true, true, TX, TY, TZ, PX, PP, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(grid4_kernel<false, true, TX, TY, TZ, PX, PP, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

cudaError_t prepare_insert_attributes() {
    cudaError_t e;
    if ((e = set_smem_shape4<8, 8, 8, 8, 68, 4>()) != cudaSuccess) return e;
    if ((e = set_smem_shape4<16, 16, 4, 17, 277, 4>()) != cudaSuccess) return e;
    if ((e = set_smem_shape4<16, 8, 8, 16, 134, 4>()) != cudaSuccess) return e;
    if ((e = set_smem_shape4<16, 16, 8, 16, 262, 2>()) != cudaSuccess) return e;
    if ((e = set_smem_shape<8, 8, 8>()) != cudaSuccess) return e;
    if ((e = set_smem_shape<16, 16, 4>()) != cudaSuccess) return e;
    if ((e = set_smem_shape<16, 8, 8>()) != cudaSuccess) return e;
    // 16 x 16 x 8 with FOM needs 5 x 2048 x 4 B per warp (160 KB for 4
    // warps); only the non-FOM variants are used
    const int smem = (int)(WARPS * 3 * 16 * 16 * 8 * sizeof(tacc_t));
    if ((e = cudaFuncSetAttribute(insert_kernel<false, true, 16, 16, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(insert_kernel<false, false, 16, 16, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

template <int TX, int TY, int TZ>
static cudaError_t launch_shape(const InsertArgs& a0, const Context& c, cudaStream_t s) {
    InsertArgs a = a0;
    const int N = c.g.map;
    a.ntx = (N + TX - 1) / TX;
    a.nty = (N + TY - 1) / TY;
    a.ntz = (N + TZ - 1) / TZ;
    const int ntiles = a.ntx * a.nty * a.ntz;
    const unsigned blocks = (unsigned)(((long)ntiles * a.R + WARPS - 1) / WARPS);
    const size_t smem = (size_t)WARPS * (c.g.fom ? 5 : 3) * TX * TY * TZ * sizeof(tacc_t);
    if (c.g.fom) {
        if (c.g.gate) insert_kernel<true, true, TX, TY, TZ><<<blocks, WARPS * 32, smem, s>>>(a);
        else insert_kernel<true, false, TX, TY, TZ><<<blocks, WARPS * 32, smem, s>>>(a);
    } else {
        if (c.g.gate) insert_kernel<false, true, TX, TY, TZ><<<blocks, WARPS * 32, smem, s>>>(a);
        else insert_kernel<false, false, TX, TY, TZ><<<blocks, WARPS * 32, smem, s>>>(a);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || a.R == 1) return e;
    if (c.g.fom) combine_kernel<true><<<148 * 8, 256, 0, s>>>(a);
    else combine_kernel<false><<<148 * 8, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <int TX, int TY, int TZ, int PX, int PP, int NW>
static cudaError_t launch_shape4(const InsertArgs& a0, const Context& c, cudaStream_t s) {
    InsertArgs a = a0;
    const int N = c.g.map;
    a.ntx = (N + TX - 1) / TX;
    a.nty = (N + TY - 1) / TY;
    a.ntz = (N + TZ - 1) / TZ;
    const int ntiles = a.ntx * a.nty * a.ntz;
    const unsigned blocks = (unsigned)(((long)ntiles * a.R + NW - 1) / NW);
    const size_t smem = (size_t)NW * PP * TZ * sizeof(float4);
    if (c.g.ewald) {
        if (c.g.gate) grid4_kernel<true, true, TX, TY, TZ, PX, PP, NW><<<blocks, NW * 32, smem, s>>>(a);
        else grid4_kernel<false, true, TX, TY, TZ, PX, PP, NW><<<blocks, NW * 32, smem, s>>>(a);
    } else {
        if (c.g.gate) grid4_kernel<true, false, TX, TY, TZ, PX, PP, NW><<<blocks, NW * 32, smem, s>>>(a);
        else grid4_kernel<false, false, TX, TY, TZ, PX, PP, NW><<<blocks, NW * 32, smem, s>>>(a);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || a.R == 1) return e;
    combine_kernel<false><<<148 * 8, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_insert(const Context& c, const float2* spectra, const DevParticle* parts, int np, int half,
                          cudaStream_t s) {
    InsertArgs a;
    a.spec = spectra;
    a.part = parts;
    a.np = np;
    a.half = half;
    a.N = c.g.map;
    a.ft = c.g.ft;
    a.pitch = c.g.ft + 2;
    a.interp = c.g.interp;
    a.maxs2 = c.g.maxs2;
    a.mins2 = c.g.mins2;
    a.mscale = c.g.mscale;
    const int h = half < 0 ? 0 : half;
    a.vol = c.d_vol[h];
    a.w = c.d_w[h];
    a.pow = c.d_pow[h];
    a.w2 = c.d_w2[h];
    a.order = c.d_tile_order;
    a.R = c.replicas;
    a.psum = c.d_part_sums;
    a.zsplit = c.g.fom ? 0 : c.zsplit;
    a.evol = c.d_evol[h];
    a.ew = c.d_ew[h];
    a.edge_rmin = c.edge_rmin;
    a.edge_rmax = c.edge_rmax;
    if (!c.g.fom) {
        switch (c.shape) {
            case 0: return launch_shape4<8, 8, 8, 8, 68, 4>(a, c, s);
            case 2: return launch_shape4<16, 8, 8, 16, 134, 4>(a, c, s);
            case 3: return launch_shape4<16, 16, 8, 16, 262, 2>(a, c, s);
            default: return launch_shape4<16, 16, 4, 17, 277, 4>(a, c, s);
        }
    }
    switch (c.shape) {
        case 0: return launch_shape<8, 8, 8>(a, c, s);
        case 2: return launch_shape<16, 8, 8>(a, c, s);
        case 3: if (!c.g.fom) return launch_shape<16, 16, 8>(a, c, s); return launch_shape<16, 16, 4>(a, c, s);
        default: return launch_shape<16, 16, 4>(a, c, s);
    }
}

}  // namespace bsg
