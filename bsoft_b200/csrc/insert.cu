// insert.cu - central-section insertion (fspace_pack_2D +
// fspace_2D_interpolate, bsoft/src/img/Bimage_reconstruct.cpp:25-174) as a
// voxel-owner gather.
//
// The reference scatters every pixel q = (h, k) of each padded particle
// transform to the map frequency m = R (h, k, 0) * inv * mscale and adds
// F(q) * w to the 1 (nearest) or 8 (trilinear) voxels around m, with index
// wrap-around, on a full complex N^3 map.  Here each thread owns one voxel v
// of the half volume z in [0, N/2] and *gathers*: for every particle of the
// batch, in order, it enumerates the pixels whose footprint covers v (and
// its wrap-around aliases v - N per axis) and accumulates in registers.
// Every voxel is written by exactly one thread per launch, so there are no
// atomics and the summation order (particle, then pixel row, then pixel) is
// fixed: results are bitwise reproducible.
//
// The same enumeration also yields the mirror voxel -v: pixel -q lands at
// -m with the same weights, so V(-v) = sum over candidates q' of v of
// F(-q') * w(q').  For interior pixels F(-q') = conj F(q') (the particle
// image is real); on the Nyquist row/column, where the reference's pixel
// grid [-ft/2, ft/2-1]^2 has no mirror partner, the value is fetched
// separately, which keeps the reference's non-Hermitian edge exact.
// Planes z = 0 and z = N/2 are their own mirrors and are computed directly.
//
// Work decomposition: a thread block owns a 16 x 16 x 4 voxel tile and each
// thread one z-column of 4 voxels, so the slab of a particle's plane cuts
// the columns of a warp alike and the lanes stay busy.  Particles whose
// plane reaches the tile are found by the whole block (256 per round) and
// compacted in order.
//
// Data movement: spectra live in HBM in a centred, padded layout
// [particle][k + ft/2][h + ft/2] of (ft + 1) x (ft + 2) complex64 values.
// For each listed particle one thread copies the particle record to shared
// memory and issues a TMA tile load (cp.async.bulk.tensor.3d, no multicast)
// of the tile's pixel footprint; a 3-stage ring of full/empty mbarriers
// lets every warp run ahead independently (no block-wide barrier per
// particle).  Footprints too large for the tile (only for unusual
// sampling) fall back to direct loads.  All waits are bounded; a wait that
// runs out sets a status word the host checks.
#include "context.cuh"

#include <cuda.h>
#include <math.h>

namespace bsg {

constexpr int BX = 16, BY = 16, BZ = 4;  // voxel tile of one thread block
constexpr int BT = BX * BY;               // one thread per z-column
constexpr int NWARPS = BT / 32;
constexpr int STAGES = 3;                 // TMA ring depth
constexpr int MAX_ITEMS = 512;            // (particle, alias) work items per round
constexpr long WAIT_LIMIT = 1L << 24;     // bounded mbarrier waits (about a second)

struct InsertArgs {
    const float2* spec;        // batch x (ft+1) x (ft+2), centred
    const DevParticle* part;   // particles of this launch
    int p_base;                // index of part[0] in the spectra buffer
    int np;
    int half;                  // only particles of this half map (-1: all)
    int N, ft, pitch;
    int interp;
    double maxs2, mins2, mscale;
    double2* vol;
    double* w;
    double* pow;
    double* w2;
    int* status;               // set non-zero if a bounded wait ran out
};

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false if the phase did not complete within the limit.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (long i = 0; i < WAIT_LIMIT; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// ---------------------------------------------------------------- geometry
// Does particle P's plane come within reach of the brick for alias
// combination a (bit i set: axis i shifted by -N)?  Bitmask over the 8.
__device__ __forceinline__ unsigned brick_mask(const DevParticle& P, int x0, int y0, int z0, int N, int ft) {
    unsigned mask = 0;
    const float ex = 0.5f * (BX - 1), ey = 0.5f * (BY - 1), ez = 0.5f * (BZ - 1);
    const float hf = 0.5f * ft;
    const float rx = hf * (fabsf(P.af[0]) + fabsf(P.bf[0])) + 1.0f;
    const float ry = hf * (fabsf(P.af[1]) + fabsf(P.bf[1])) + 1.0f;
    const float rz = hf * (fabsf(P.af[2]) + fabsf(P.bf[2])) + 1.0f;
    const float n0 = (float)P.nrm[0], n1 = (float)P.nrm[1], n2 = (float)P.nrm[2];
    const float slack = P.slab + fabsf(n0) * ex + fabsf(n1) * ey + fabsf(n2) * ez + 1e-3f;
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

// Pixel bounding box [h_lo, h_hi] x [k_lo, k_hi] of every pixel whose tent
// reaches the brick alias box (brick expanded by one voxel).
__device__ __forceinline__ void brick_footprint(const DevParticle& P, int x0, int y0, int z0, int hf,
                                                int& h_lo, int& h_hi, int& k_lo, int& k_hi) {
    const double E[3] = {0.5 * (BX - 1) + 1.0, 0.5 * (BY - 1) + 1.0, 0.5 * (BZ - 1) + 1.0};
    const double C[3] = {x0 + 0.5 * (BX - 1), y0 + 0.5 * (BY - 1), z0 + 0.5 * (BZ - 1)};
    const double st2 = (double)P.step * (double)P.step;
    double uc = 0, vc = 0, hu = 0, hv = 0;
    for (int i = 0; i < 3; ++i) {
        uc += P.ad[i] * C[i];
        vc += P.bd[i] * C[i];
        hu += fabs(P.ad[i]) * E[i];
        hv += fabs(P.bd[i]) * E[i];
    }
    uc /= st2; vc /= st2; hu /= st2; hv /= st2;
    h_lo = max((int)ceil(uc - hu) - 1, -hf);
    h_hi = min((int)floor(uc + hu) + 1, hf);
    k_lo = max((int)ceil(vc - hv) - 1, -hf);
    k_hi = min((int)floor(vc + hv) + 1, hf);
}

struct Acc {
    float2 v, m;      // voxel and mirror complex sums (one particle)
    float w, wm;
    float p, pm;
    float q, qm;
};

struct AccD {
    double vx, vy, mx, my, w, wm, p, pm, q, qm;
};

template <bool FOM>
__device__ __forceinline__ void fold(AccD& d, const Acc& a, bool mirror) {
    d.vx += a.v.x; d.vy += a.v.y; d.w += a.w;
    if (FOM) { d.p += a.p; d.q += a.q; }
    if (mirror) {
        d.mx += a.m.x; d.my += a.m.y; d.wm += a.wm;
        if (FOM) { d.pm += a.pm; d.qm += a.qm; }
    }
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

// Pixel source: a shared-memory tile (origin c0, r0 in centred coordinates)
// with a direct-load fallback for pixels outside it.
struct Src {
    const float2* tile;     // nullptr: direct loads only
    int c0, r0, tw;
    const float2* g;        // this particle's centred spectrum
    int pitch, hf;
    __device__ __forceinline__ float2 get(int h, int k) const {
        const int c = h + hf, r = k + hf;
        if (tile) {
            const int lc = c - c0, lr = r - r0;
            if ((unsigned)lc < (unsigned)tw && (unsigned)lr < (unsigned)tw) return tile[lr * tw + lc];
        }
        return __ldg(g + (size_t)r * pitch + c);
    }
    __device__ __forceinline__ float2 get_global(int h, int k) const {
        return __ldg(g + (size_t)(k + hf) * pitch + (h + hf));
    }
};

// Accumulate candidate pixel (h, k) with weight wt: into the voxel if the
// pixel is on the reference grid, into the mirror if -q is.
template <bool FOM>
__device__ __forceinline__ void accumulate(const Src& S, int h, int k, float wt, bool own, bool mir,
                                           bool mirror, int hf, Acc& acc) {
    const bool interior = (h > -hf) & (h < hf) & (k > -hf) & (k < hf);
    const bool inG = own && h != hf && k != hf;
    float2 f = make_float2(0.f, 0.f);
    if (inG || (mirror && mir && interior)) f = S.get(h, k);
    if (inG) {
        acc.v.x = fmaf(f.x, wt, acc.v.x);
        acc.v.y = fmaf(f.y, wt, acc.v.y);
        acc.w += wt;
        if (FOM) { acc.p = fmaf(wt, f.x * f.x + f.y * f.y, acc.p); acc.q = fmaf(wt, wt, acc.q); }
    }
    if (mirror && mir && h != -hf && k != -hf) {
        float2 g;
        if (interior) g = make_float2(f.x, -f.y);        // F(-q) = conj F(q)
        else g = S.get_global(-h, -k);                    // Nyquist edge: the reference's own value
        acc.m.x = fmaf(g.x, wt, acc.m.x);
        acc.m.y = fmaf(g.y, wt, acc.m.y);
        acc.wm += wt;
        if (FOM) { acc.pm = fmaf(wt, g.x * g.x + g.y * g.y, acc.pm); acc.qm = fmaf(wt, wt, acc.qm); }
    }
}

template <bool FOM, bool GATE>
__device__ __forceinline__ void gather_trilinear(const InsertArgs& a, const DevParticle& P, const Src& S,
                                                 double cxd, double cyd, double czd, double t, bool mirror,
                                                 Acc& acc) {
    const int hf = a.ft / 2;
    // plane coordinates (pixels) of the voxel's projection
    const double u = (P.ad[0] * cxd + P.ad[1] * cyd + P.ad[2] * czd) * P.inv_st2;
    const double v = (P.bd[0] * cxd + P.bd[1] * cyd + P.bd[2] * czd) * P.inv_st2;
    const int h0 = (int)rint(u), k0 = (int)rint(v);
    // offsets of pixel (h0, k0) from the voxel in double, then float steps
    const float d0x = (float)(h0 * P.ad[0] + k0 * P.bd[0] - cxd);
    const float d0y = (float)(h0 * P.ad[1] + k0 * P.bd[1] - cyd);
    const float d0z = (float)(h0 * P.ad[2] + k0 * P.bd[2] - czd);
    const float ax = P.af[0], ay = P.af[1], az = P.af[2];
    const float bx = P.bf[0], by = P.bf[1], bz = P.bf[2];
    const float ibx = P.ib[0], iby = P.ib[1], ibz = P.ib[2];
    const float rad = sqrtf(fmaxf(0.f, 3.f - (float)(t * t))) * P.inv_step;
    const float uu = (float)(u - h0);
    const int dh0 = max((int)ceilf(uu - rad), -hf - h0);
    const int dh1 = min((int)floorf(uu + rad), hf - h0);
    for (int dh = dh0; dh <= dh1; ++dh) {
        const float ex = fmaf((float)dh, ax, d0x);
        const float ey = fmaf((float)dh, ay, d0y);
        const float ez = fmaf((float)dh, az, d0z);
        float lo = -1e30f, hi = 1e30f;
        if (ibx != 0.f) { float p = (-1.f - ex) * ibx, q = (1.f - ex) * ibx; lo = fmaxf(lo, fminf(p, q)); hi = fminf(hi, fmaxf(p, q)); }
        else if (fabsf(ex) >= 1.f) continue;
        if (iby != 0.f) { float p = (-1.f - ey) * iby, q = (1.f - ey) * iby; lo = fmaxf(lo, fminf(p, q)); hi = fminf(hi, fmaxf(p, q)); }
        else if (fabsf(ey) >= 1.f) continue;
        if (ibz != 0.f) { float p = (-1.f - ez) * ibz, q = (1.f - ez) * ibz; lo = fmaxf(lo, fminf(p, q)); hi = fminf(hi, fmaxf(p, q)); }
        else if (fabsf(ez) >= 1.f) continue;
        const int dk0 = max((int)ceilf(lo), -hf - k0);
        const int dk1 = min((int)floorf(hi), hf - k0);
        const int h = h0 + dh;
        for (int dk = dk0; dk <= dk1; ++dk) {
            const float fx = fmaf((float)dk, bx, ex);
            const float fy = fmaf((float)dk, by, ey);
            const float fz = fmaf((float)dk, bz, ez);
            float wt = fmaxf(0.f, 1.f - fabsf(fx)) * fmaxf(0.f, 1.f - fabsf(fy)) * fmaxf(0.f, 1.f - fabsf(fz));
            const int k = k0 + dk;
            wt *= P.pw;
            if (GATE) {
                bool keep;
                const float tw = pixel_weight_gate(a, P, h, k, keep);
                if (!keep) continue;
                wt *= tw;
            }
            accumulate<FOM>(S, h, k, wt, true, true, mirror, hf, acc);
        }
    }
}

// Nearest / weighted-nearest: pixel q goes to round(m) (floor(m + 0.5) of a
// double m in fspace_2D_interpolate); decisions in double.
template <bool FOM, bool GATE>
__device__ __forceinline__ void gather_nearest(const InsertArgs& a, const DevParticle& P, const Src& S,
                                               double cx, double cy, double cz, double t, bool mirror,
                                               bool weighted, Acc& acc) {
    const int hf = a.ft / 2;
    const double u = (P.ad[0] * cx + P.ad[1] * cy + P.ad[2] * cz) * P.inv_st2;
    const double v = (P.bd[0] * cx + P.bd[1] * cy + P.bd[2] * cz) * P.inv_st2;
    const double rad = sqrt(fmax(0.0, 0.75 - t * t)) * P.inv_step + 1e-9;
    const int hlo = max((int)ceil(u - rad), -hf), hhi = min((int)floor(u + rad), hf);
    const int klo = max((int)ceil(v - rad), -hf), khi = min((int)floor(v + rad), hf);
    for (int h = hlo; h <= hhi; ++h) {
        for (int k = klo; k <= khi; ++k) {
            const double dx = h * P.ad[0] + k * P.bd[0] - cx;
            const double dy = h * P.ad[1] + k * P.bd[1] - cy;
            const double dz = h * P.ad[2] + k * P.bd[2] - cz;
            // voxel side: floor(m + 0.5) == c  <=>  -0.5 <= d < 0.5
            const bool own = dx >= -0.5 && dx < 0.5 && dy >= -0.5 && dy < 0.5 && dz >= -0.5 && dz < 0.5;
            // mirror side: floor(-m + 0.5) == -c  <=>  -0.5 < d <= 0.5
            const bool mir = dx > -0.5 && dx <= 0.5 && dy > -0.5 && dy <= 0.5 && dz > -0.5 && dz <= 0.5;
            if (!own && !mir) continue;
            float wt = P.pw;
            if (GATE) {
                bool keep;
                const float tw = pixel_weight_gate(a, P, h, k, keep);
                if (!keep) continue;
                wt *= tw;
            }
            float w = wt;
            if (weighted) w = (float)((double)wt * (1.0 - sqrt(dx * dx + dy * dy + dz * dz)));
            if (!(w > 0.f)) continue;
            accumulate<FOM>(S, h, k, w, own, mir, mirror, hf, acc);
        }
    }
}

// One particle (alias `al`) against this thread's column of BZ voxels.
template <bool FOM, bool GATE>
__device__ __forceinline__ void gather_column(const InsertArgs& a, const DevParticle& P, const Src& S, int x,
                                              int y, int z0, int al, AccD* acc) {
    const int N = a.N;
    if (x >= N || y >= N) return;
    const double cx = (double)(x - ((al & 1) ? N : 0));
    const double cy = (double)(y - ((al & 2) ? N : 0));
    const double czb = (double)(z0 - ((al & 4) ? N : 0));
    const double tb = P.nrm[0] * cx + P.nrm[1] * cy + P.nrm[2] * czb;
    const double reach = a.interp == 2 ? (double)P.slab : 0.5 * P.slab + 1e-9;
#pragma unroll
    for (int iz = 0; iz < BZ; ++iz) {
        const int z = z0 + iz;
        const double t = tb + P.nrm[2] * iz;
        if (z > N / 2 || !(fabs(t) < reach || (a.interp != 2 && fabs(t) <= reach))) continue;
        const bool mirror = z > 0 && z < N / 2;
        Acc part = {};
        if (a.interp == 2) gather_trilinear<FOM, GATE>(a, P, S, cx, cy, czb + iz, t, mirror, part);
        else gather_nearest<FOM, GATE>(a, P, S, cx, cy, czb + iz, t, mirror, a.interp == 1, part);
        fold<FOM>(acc[iz], part, mirror);
    }
}

template <bool FOM, bool GATE, int TW>
__global__ void __launch_bounds__(BT, FOM ? 1 : 2) insert_kernel(InsertArgs a, const __grid_constant__ CUtensorMap tmap) {
    const int N = a.N, hf = a.ft / 2;
    const int cxl = threadIdx.x % BX, cyl = threadIdx.x / BX;
    const int x0 = blockIdx.x * BX, y0 = blockIdx.y * BY, z0 = blockIdx.z * BZ;
    const int x = x0 + cxl, y = y0 + cyl;
    const size_t spec_stride = (size_t)(2 * hf + 1) * a.pitch;

    extern __shared__ __align__(128) float2 s_dyn[];      // STAGES x TW x TW pixel tiles
    __shared__ __align__(16) DevParticle s_part[STAGES];
    __shared__ int s_meta[STAGES][4];                     // c0, r0, fits, particle index
    __shared__ __align__(8) uint64_t s_full[STAGES];
    __shared__ __align__(8) uint64_t s_empty[STAGES];
    __shared__ unsigned s_list[BT];
    __shared__ unsigned short s_item[MAX_ITEMS];          // (list entry << 3) | alias
    __shared__ int s_warp[NWARPS + 1];
    __shared__ int s_nitems;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) { mbar_init(&s_full[s], 1); mbar_init(&s_empty[s], NWARPS); }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    bool failed = false;
    AccD acc[BZ];
#pragma unroll
    for (int i = 0; i < BZ; ++i) acc[i] = AccD{};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long g = 0;                                           // items started before this round

    // producer step (thread 0): item `it` of this round, global number gi
    auto produce = [&](int it, long gi, int base) {
        const int st = (int)(gi % STAGES);
        const long use = gi / STAGES;
        if (use >= 1 && !failed && !mbar_wait(&s_empty[st], (uint32_t)((use - 1) & 1))) failed = true;
        const unsigned item = s_item[it];
        const int pi = base + (int)(s_list[item >> 3] & 0xffffu);
        const int al = item & 7;
        const DevParticle& P = a.part[pi];
        s_part[st] = P;
        int hl, hh, kl, kh;
        brick_footprint(P, x0 - ((al & 1) ? N : 0), y0 - ((al & 2) ? N : 0), z0 - ((al & 4) ? N : 0), hf,
                        hl, hh, kl, kh);
        const int c0 = (hl + hf) & ~1;                    // 16-byte aligned x coordinate
        const int r0 = kl + hf;
        const bool fits = (hh + hf - c0 < TW) && (kh + hf - r0 < TW);
        s_meta[st][0] = c0;
        s_meta[st][1] = r0;
        s_meta[st][2] = fits ? 1 : 0;
        s_meta[st][3] = pi;
        if (fits && !failed) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&s_full[st], (uint32_t)(TW * TW * sizeof(float2)));
            tma_load_3d(s_dyn + (size_t)st * TW * TW, &tmap, c0, r0, a.p_base + pi, &s_full[st]);
        } else {
            if (!fits) s_meta[st][2] = 0;
            mbar_arrive(&s_full[st]);
        }
    };

    for (int base = 0; base < a.np; base += BT) {
        const int p = base + threadIdx.x;
        unsigned mask = 0;
        if (p < a.np) {
            const DevParticle& P = a.part[p];
            if (P.half == a.half || a.half < 0) mask = brick_mask(P, x0, y0, z0, N, a.ft);
        }
        // ordered compaction of (particle, alias mask)
        const unsigned ball = __ballot_sync(0xffffffffu, mask != 0);
        const int before = __popc(ball & ((1u << lane) - 1));
        if (lane == 0) s_warp[warp] = __popc(ball);
        __syncthreads();
        if (threadIdx.x == 0) {
            int run = 0;
            for (int w = 0; w < NWARPS; ++w) { const int c = s_warp[w]; s_warp[w] = run; run += c; }
            s_warp[NWARPS] = run;
        }
        __syncthreads();
        if (mask) s_list[s_warp[warp] + before] = (unsigned)threadIdx.x | (mask << 16);
        __syncthreads();
        if (threadIdx.x == 0) {
            int n = 0;
            const int cnt = s_warp[NWARPS];
            for (int e = 0; e < cnt; ++e) {
                const unsigned am = s_list[e] >> 16;
                for (int al = 0; al < 8; ++al)
                    if ((am >> al) & 1u) {
                        if (n < MAX_ITEMS) s_item[n] = (unsigned short)((e << 3) | al);
                        ++n;
                    }
            }
            s_nitems = n;
        }
        __syncthreads();
        const int nitems = s_nitems;
        if (nitems > MAX_ITEMS) {
            // more items than the list holds (not reached for supported
            // sizes): a direct-load pass over this round's entries
            const int cnt = s_warp[NWARPS];
            for (int e = 0; e < cnt; ++e) {
                const unsigned ent = s_list[e];
                const int pi = base + (int)(ent & 0xffffu);
                const Src S{nullptr, 0, 0, TW, a.spec + (size_t)(a.p_base + pi) * spec_stride, a.pitch, hf};
                for (int al = 0; al < 8; ++al)
                    if ((ent >> (16 + al)) & 1u) gather_column<FOM, GATE>(a, a.part[pi], S, x, y, z0, al, acc);
            }
            __syncthreads();
            continue;
        }
        if (threadIdx.x == 0)
            for (int j = 0; j < STAGES - 1 && j < nitems; ++j) produce(j, g + j, base);
        for (int it = 0; it < nitems; ++it) {
            if (threadIdx.x == 0 && it + STAGES - 1 < nitems) produce(it + STAGES - 1, g + it + STAGES - 1, base);
            const long gi = g + it;
            const int st = (int)(gi % STAGES);
            if (!failed && !mbar_wait(&s_full[st], (uint32_t)((gi / STAGES) & 1))) failed = true;
            if (!failed) {
                const DevParticle& P = s_part[st];
                const int pi = s_meta[st][3];
                const Src S{s_meta[st][2] ? s_dyn + (size_t)st * TW * TW : nullptr, s_meta[st][0], s_meta[st][1],
                            TW, a.spec + (size_t)(a.p_base + pi) * spec_stride, a.pitch, hf};
                gather_column<FOM, GATE>(a, P, S, x, y, z0, s_item[it] & 7, acc);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&s_empty[st]);
        }
        g += nitems;
        __syncthreads();
    }
    if (failed) {
        // a tile never arrived: report it and give copies still in flight a
        // bounded chance to land before the block's shared memory is released
        if (threadIdx.x == 0) atomicExch(a.status, 1);
        for (int s = 0; s < STAGES; ++s) {
            const long last = g - 1 - ((g - 1 - s) % STAGES + STAGES) % STAGES;   // last item on stage s
            if (g > 0 && last >= 0) mbar_wait(&s_full[s], (uint32_t)((last / STAGES) & 1));
        }
        return;
    }
    if (x >= N || y >= N) return;
#pragma unroll
    for (int iz = 0; iz < BZ; ++iz) {
        const int z = z0 + iz;
        if (z > N / 2) break;
        const AccD& c = acc[iz];
        const size_t idx = ((size_t)z * N + y) * N + x;
        double2 o = a.vol[idx];
        a.vol[idx] = make_double2(o.x + c.vx, o.y + c.vy);
        a.w[idx] += c.w;
        if (FOM) { a.pow[idx] += c.p; a.w2[idx] += c.q; }
        if (z > 0 && z < N / 2) {
            const size_t midx = ((size_t)((N - z) % N) * N + (N - y) % N) * N + (N - x) % N;
            double2 om = a.vol[midx];
            a.vol[midx] = make_double2(om.x + c.mx, om.y + c.my);
            a.w[midx] += c.wm;
            if (FOM) { a.pow[midx] += c.pm; a.w2[midx] += c.qm; }
        }
    }
}

template <int TW>
static cudaError_t launch_tw(const InsertArgs& a, const CUtensorMap& map, bool fom, bool gate, dim3 grid,
                             cudaStream_t s) {
    const size_t smem = STAGES * sizeof(float2) * TW * TW;
    if (fom) {
        if (gate) insert_kernel<true, true, TW><<<grid, BT, smem, s>>>(a, map);
        else insert_kernel<true, false, TW><<<grid, BT, smem, s>>>(a, map);
    } else {
        if (gate) insert_kernel<false, true, TW><<<grid, BT, smem, s>>>(a, map);
        else insert_kernel<false, false, TW><<<grid, BT, smem, s>>>(a, map);
    }
    return cudaGetLastError();
}

template <int TW>
static cudaError_t set_smem_tw() {
    const int smem = (int)(STAGES * sizeof(float2) * TW * TW);
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(insert_kernel<true, true, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(insert_kernel<true, false, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(insert_kernel<false, true, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(insert_kernel<false, false, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

cudaError_t prepare_insert_attributes() {
    cudaError_t e = set_smem_tw<32>();
    if (e != cudaSuccess) return e;
    return set_smem_tw<64>();
}

// Edge of the square pixel tile that always holds a voxel tile's footprint
// at this voxels-per-pixel step (brick_footprint, widest orientation).
int tile_edge_for_step(double step) {
    const double E = sqrt(pow(0.5 * (BX - 1) + 1.0, 2) + pow(0.5 * (BY - 1) + 1.0, 2) + pow(0.5 * (BZ - 1) + 1.0, 2));
    const int need = (int)ceil(2.0 * E / step) + 4;      // +2 rounding, +1 alignment, +1 inclusive
    return need <= 32 ? 32 : need <= 64 ? 64 : 0;
}

cudaError_t launch_insert(const Context& c, const float2* spectra, int p0, int np, int half, cudaStream_t s) {
    InsertArgs a;
    a.spec = spectra;
    a.part = c.d_part + p0;
    a.p_base = p0;
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
    a.status = c.d_status;
    const int N = c.g.map;
    dim3 grid((N + BX - 1) / BX, (N + BY - 1) / BY, (N / 2 + 1 + BZ - 1) / BZ);
    // larger footprints than 64 (very fine sampling) use the 64 tile with
    // direct loads for the pixels outside it
    if (c.tile_edge == 32) return launch_tw<32>(a, c.spec_map[0], c.g.fom, c.g.gate, grid, s);
    return launch_tw<64>(a, c.spec_map[1], c.g.fom, c.g.gate, grid, s);
}

}  // namespace bsg
