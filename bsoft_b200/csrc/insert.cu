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
// F(-q') * w(q').  Membership of q' and -q' in the pixel grid
// [-ft/2, ft/2-1]^2 is tested separately, which keeps the reference's
// non-Hermitian Nyquist row/column exact.  Planes z = 0 and z = N/2 are
// their own mirrors and are computed directly.
//
// Thread block = 8 x 8 x 4 voxel brick.  Particles are tested against the
// brick (plane slab and reach, per alias) by the whole block in chunks of
// 256 and compacted, in order, into a shared list.
#include "context.cuh"

#include <math.h>

namespace bsg {

constexpr int BX = 8, BY = 8, BZ = 4;
constexpr int BT = BX * BY * BZ;

struct InsertArgs {
    const float2* spec;        // np x ft x ft
    const DevParticle* part;   // np
    int np;
    int half;                  // only particles of this half map
    int N, ft;
    int interp;
    int gate;                  // 1: test the s^2 window / taper per pixel
    double maxs2, mins2, mscale;
    double2* vol;
    double* w;
    double* pow;
    double* w2;
};

// Does particle P's plane come within reach of the brick for alias combination
// (ax, ay, az)?  Returns a bitmask over the 8 alias combinations.
__device__ __forceinline__ unsigned brick_mask(const DevParticle& P, int x0, int y0, int z0, int N, int ft) {
    unsigned mask = 0;
    const float ex = 0.5f * (BX - 1), ey = 0.5f * (BY - 1), ez = 0.5f * (BZ - 1);
    const float hf = 0.5f * ft;
    // reach of the pixel square along each axis, plus the tent support
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

// Per (voxel, particle) partial sums in float (a handful of terms each)...
struct Acc {
    float2 v, m;      // voxel and mirror complex sums
    float w, wm;      // weights
    float p, pm;      // power (fom)
    float q, qm;      // weight^2 (fom)
};

// ... folded into the per-voxel running sums over the batch in double.
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
    // s2 exactly as fspace_pack_2D forms it: s = (h, k) * inv (double)
    const double inv = sqrt(P.inv2);
    const double sx = h * inv, sy = k * inv;
    const double s2 = sx * sx + sy * sy;
    keep = (s2 >= a.mins2 && s2 <= a.maxs2);
    const double d = (a.maxs2 - s2) * a.mscale;
    return d < 1.0 ? (float)sqrt(d > 0 ? d : 0.0) : 1.0f;
}

template <bool FOM, bool GATE>
__device__ __forceinline__ void gather_trilinear(const InsertArgs& a, const DevParticle& P, const float2* __restrict__ S,
                                                 float cx, float cy, float cz, bool mirror, Acc& acc) {
    const int ft = a.ft, hf = ft / 2, fm = ft - 1;
    // distance to the plane and reach test for this voxel alias
    const double cxd = cx, cyd = cy, czd = cz;
    const double t = P.nrm[0] * cxd + P.nrm[1] * cyd + P.nrm[2] * czd;
    if (fabs(t) >= (double)P.slab) return;
    // plane coordinates (pixels) of the projection of c
    const double st2 = (double)P.step * (double)P.step;
    const double u = (P.ad[0] * cxd + P.ad[1] * cyd + P.ad[2] * czd) / st2;
    const double v = (P.bd[0] * cxd + P.bd[1] * cyd + P.bd[2] * czd) / st2;
    const int h0 = (int)rint(u), k0 = (int)rint(v);
    // local offsets of pixel (h0, k0) from c, in double, then float increments
    const float d0x = (float)(h0 * P.ad[0] + k0 * P.bd[0] - cxd);
    const float d0y = (float)(h0 * P.ad[1] + k0 * P.bd[1] - cyd);
    const float d0z = (float)(h0 * P.ad[2] + k0 * P.bd[2] - czd);
    const float ax = P.af[0], ay = P.af[1], az = P.af[2];
    const float bx = P.bf[0], by = P.bf[1], bz = P.bf[2];
    const float rad = sqrtf(fmaxf(0.f, 3.f - (float)(t * t))) / P.step;
    const float uu = (float)(u - h0);
    int dh0 = (int)ceilf(uu - rad), dh1 = (int)floorf(uu + rad);
    dh0 = max(dh0, -hf - h0);
    dh1 = min(dh1, hf - h0);
    const float ibx = fabsf(bx) > 1e-6f ? 1.f / bx : 0.f;
    const float iby = fabsf(by) > 1e-6f ? 1.f / by : 0.f;
    const float ibz = fabsf(bz) > 1e-6f ? 1.f / bz : 0.f;
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
        int dk0 = (int)ceilf(lo), dk1 = (int)floorf(hi);
        dk0 = max(dk0, -hf - k0);
        dk1 = min(dk1, hf - k0);
        const int h = h0 + dh;
        const bool hin = (h != hf), hmin = (h != -hf);
        const float2* rowbase = S + (h & fm);
        const float2* mrowbase = S + ((-h) & fm);
        for (int dk = dk0; dk <= dk1; ++dk) {
            const float fx = fmaf((float)dk, bx, ex);
            const float fy = fmaf((float)dk, by, ey);
            const float fz = fmaf((float)dk, bz, ez);
            float wt = fmaxf(0.f, 1.f - fabsf(fx)) * fmaxf(0.f, 1.f - fabsf(fy)) * fmaxf(0.f, 1.f - fabsf(fz));
            const int k = k0 + dk;
            wt *= P.pw;
            if (GATE) {
                bool keep;
                float tw = pixel_weight_gate(a, P, h, k, keep);
                if (!keep) continue;
                wt *= tw;
            }
            if (hin && k != hf) {
                const float2 f = __ldg(rowbase + (size_t)(k & fm) * ft);
                acc.v.x = fmaf(f.x, wt, acc.v.x);
                acc.v.y = fmaf(f.y, wt, acc.v.y);
                acc.w += wt;
                if (FOM) { acc.p = fmaf(wt, f.x * f.x + f.y * f.y, acc.p); acc.q = fmaf(wt, wt, acc.q); }
            }
            if (mirror && hmin && k != -hf) {
                const float2 f = __ldg(mrowbase + (size_t)((-k) & fm) * ft);
                acc.m.x = fmaf(f.x, wt, acc.m.x);
                acc.m.y = fmaf(f.y, wt, acc.m.y);
                acc.wm += wt;
                if (FOM) { acc.pm = fmaf(wt, f.x * f.x + f.y * f.y, acc.pm); acc.qm = fmaf(wt, wt, acc.qm); }
            }
        }
    }
}

// Nearest / weighted-nearest: pixel q goes to round(m).  Decisions in double
// (fspace_2D_interpolate rounds floor(m + 0.5) of a double m).
template <bool FOM, bool GATE>
__device__ __forceinline__ void gather_nearest(const InsertArgs& a, const DevParticle& P, const float2* __restrict__ S,
                                               double cx, double cy, double cz, bool mirror, bool weighted, Acc& acc) {
    const int ft = a.ft, hf = ft / 2, fm = ft - 1;
    const double t = P.nrm[0] * cx + P.nrm[1] * cy + P.nrm[2] * cz;
    if (fabs(t) > 0.5 * P.slab + 1e-9) return;
    const double st2 = (double)P.step * (double)P.step;
    const double u = (P.ad[0] * cx + P.ad[1] * cy + P.ad[2] * cz) / st2;
    const double v = (P.bd[0] * cx + P.bd[1] * cy + P.bd[2] * cz) / st2;
    const double rad = sqrt(fmax(0.0, 0.75 - t * t)) / P.step + 1e-9;
    const int hlo = max((int)ceil(u - rad), -hf), hhi = min((int)floor(u + rad), hf);
    const int klo = max((int)ceil(v - rad), -hf), khi = min((int)floor(v + rad), hf);
    for (int h = hlo; h <= hhi; ++h) {
        for (int k = klo; k <= khi; ++k) {
            const double mx = h * P.ad[0] + k * P.bd[0];
            const double my = h * P.ad[1] + k * P.bd[1];
            const double mz = h * P.ad[2] + k * P.bd[2];
            const double dx = mx - cx, dy = my - cy, dz = mz - cz;
            float wt = P.pw;
            if (GATE) {
                bool keep;
                float tw = pixel_weight_gate(a, P, h, k, keep);
                if (!keep) continue;
                wt *= tw;
            }
            // voxel side: floor(m + 0.5) == c  <=>  -0.5 <= d < 0.5
            const bool own = dx >= -0.5 && dx < 0.5 && dy >= -0.5 && dy < 0.5 && dz >= -0.5 && dz < 0.5;
            // mirror side: floor(-m + 0.5) == -c  <=>  -0.5 < d <= 0.5
            const bool mir = dx > -0.5 && dx <= 0.5 && dy > -0.5 && dy <= 0.5 && dz > -0.5 && dz <= 0.5;
            float w = wt;
            if (weighted) w = (float)((double)wt * (1.0 - sqrt(dx * dx + dy * dy + dz * dz)));
            if (!(w > 0.f)) continue;
            if (own && h != hf && k != hf) {
                const float2 f = __ldg(S + (size_t)(k & fm) * ft + (h & fm));
                acc.v.x = fmaf(f.x, w, acc.v.x);
                acc.v.y = fmaf(f.y, w, acc.v.y);
                acc.w += w;
                if (FOM) { acc.p = fmaf(w, f.x * f.x + f.y * f.y, acc.p); acc.q = fmaf(w, w, acc.q); }
            }
            if (mirror && mir && h != -hf && k != -hf) {
                const float2 f = __ldg(S + (size_t)((-k) & fm) * ft + ((-h) & fm));
                acc.m.x = fmaf(f.x, w, acc.m.x);
                acc.m.y = fmaf(f.y, w, acc.m.y);
                acc.wm += w;
                if (FOM) { acc.pm = fmaf(w, f.x * f.x + f.y * f.y, acc.pm); acc.qm = fmaf(w, w, acc.qm); }
            }
        }
    }
}

template <bool FOM, bool GATE>
__global__ void __launch_bounds__(BT, 2) insert_kernel(InsertArgs a) {
    const int N = a.N;
    const int tx = threadIdx.x % BX, ty = (threadIdx.x / BX) % BY, tz = threadIdx.x / (BX * BY);
    const int x0 = blockIdx.x * BX, y0 = blockIdx.y * BY, z0 = blockIdx.z * BZ;
    const int x = x0 + tx, y = y0 + ty, z = z0 + tz;
    const bool valid = x < N && y < N && z <= N / 2;
    const bool mirror = valid && z > 0 && z < N / 2;

    __shared__ unsigned s_list[BT];
    __shared__ int s_warp[BT / 32 + 1];
    AccD acc = {};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

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
            for (int w = 0; w < BT / 32; ++w) { int c = s_warp[w]; s_warp[w] = run; run += c; }
            s_warp[BT / 32] = run;
        }
        __syncthreads();
        if (mask) s_list[s_warp[warp] + before] = (unsigned)threadIdx.x | (mask << 16);
        __syncthreads();
        const int cnt = s_warp[BT / 32];
        for (int e = 0; e < cnt; ++e) {
            const unsigned ent = s_list[e];
            const int pi = base + (int)(ent & 0xffffu);
            const unsigned am = ent >> 16;
            if (!valid) continue;
            const DevParticle& P = a.part[pi];
            const float2* S = a.spec + (size_t)pi * a.ft * a.ft;
            Acc part = {};
            for (int al = 0; al < 8; ++al) {
                if (!(am & (1u << al))) continue;
                const float cx = (float)(x - ((al & 1) ? N : 0));
                const float cy = (float)(y - ((al & 2) ? N : 0));
                const float cz = (float)(z - ((al & 4) ? N : 0));
                if (a.interp == 2) gather_trilinear<FOM, GATE>(a, P, S, cx, cy, cz, mirror, part);
                else gather_nearest<FOM, GATE>(a, P, S, cx, cy, cz, mirror, a.interp == 1, part);
            }
            fold<FOM>(acc, part, mirror);
        }
        __syncthreads();
    }
    if (!valid) return;
    const size_t idx = ((size_t)z * N + y) * N + x;
    double2 o = a.vol[idx];
    a.vol[idx] = make_double2(o.x + acc.vx, o.y + acc.vy);
    a.w[idx] += acc.w;
    if (FOM) { a.pow[idx] += acc.p; a.w2[idx] += acc.q; }
    if (mirror) {
        const size_t midx = ((size_t)((N - z) % N) * N + (N - y) % N) * N + (N - x) % N;
        double2 om = a.vol[midx];
        a.vol[midx] = make_double2(om.x + acc.mx, om.y + acc.my);
        a.w[midx] += acc.wm;
        if (FOM) { a.pow[midx] += acc.pm; a.w2[midx] += acc.qm; }
    }
}

cudaError_t launch_insert(const Context& c, const float2* spectra, int p0, int np, int half, cudaStream_t s) {
    InsertArgs a;
    a.spec = spectra + (size_t)p0 * c.g.ft * c.g.ft;
    a.part = c.d_part + p0;
    a.np = np;
    a.half = half;
    a.N = c.g.map;
    a.ft = c.g.ft;
    a.interp = c.g.interp;
    a.maxs2 = c.g.maxs2;
    a.mins2 = c.g.mins2;
    a.mscale = c.g.mscale;
    const int h = half < 0 ? 0 : half;
    a.vol = c.d_vol[h];
    a.w = c.d_w[h];
    a.pow = c.d_pow[h];
    a.w2 = c.d_w2[h];
    // per-pixel s^2 window / taper test only when the run's limits can bite
    a.gate = c.g.gate;
    const int N = c.g.map;
    dim3 grid((N + BX - 1) / BX, (N + BY - 1) / BY, (N / 2 + 1 + BZ - 1) / BZ);
    if (c.g.fom) {
        if (a.gate) insert_kernel<true, true><<<grid, BT, 0, s>>>(a);
        else insert_kernel<true, false><<<grid, BT, 0, s>>>(a);
    } else {
        if (a.gate) insert_kernel<false, true><<<grid, BT, 0, s>>>(a);
        else insert_kernel<false, false><<<grid, BT, 0, s>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace bsg
