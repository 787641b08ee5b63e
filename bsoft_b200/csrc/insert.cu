// insert.cu - central-section insertion (fspace_pack_2D +
// fspace_2D_interpolate, bsoft/src/img/Bimage_reconstruct.cpp:25-174).
//
// The reference scatters every pixel q = (h, k) of each padded particle
// transform, q in [-ft/2, ft/2-1]^2, to the map frequency
// m = R (h, k, 0) * inv * mscale and adds F(q) * w to the 1 (nearest) or 8
// (trilinear) voxels around m, with index wrap-around, on a full complex
// N^3 map, plus w to the weight map (and w |F|^2, w^2 to the FOM channels).
//
// Here a thread block owns a 16 x 16 x 4 tile of the map and keeps its sums
// in shared memory for the whole batch.  Particles whose plane (or one of
// its wrap-around aliases) reaches the tile are found by the block, 256 at a
// time, and compacted in order; the warps then walk those particles' pixel
// footprints row by row (lanes along h, so spectrum reads are coalesced) and
// add each pixel's contributions to the tile.
//
// Determinism: the shared sums are 64-bit fixed point.  Each contribution
// is the float product F * w exactly as computed, scaled by a power of two
// chosen per batch so that the largest possible |F * w| is below 2^44, and
// added with an integer atomic.  Integer addition is associative, so every
// schedule gives bitwise the same sums; the quantum (2^-44 of the batch's
// largest term) is far below float resolution.  At the end of the batch the
// tile is converted to double and added to the FP64 accumulators in HBM
// (each voxel belongs to exactly one block).
#include "context.cuh"

#include <math.h>

namespace bsg {

constexpr int TX = 16, TY = 16, TZ = 4;   // map tile of one thread block
constexpr int TV = TX * TY * TZ;          // voxels per tile
constexpr int NT = 256;                   // threads per block
constexpr int NWARPS = NT / 32;

struct InsertArgs {
    const float2* spec;        // batch x (ft+1) x (ft+2), centred
    const DevParticle* part;   // particles of this launch
    int p_base;                // index of part[0] in the spectra buffer
    int np;
    int half;                  // only particles of this half map (-1: all)
    int N, ft, pitch;
    int interp;
    double maxs2, mins2, mscale;
    const unsigned* fmax_bits; // batch max of |Re F|, |Im F| (float bits)
    float pw_max;              // batch max particle weight
    int fix_bits;              // largest |F w| maps below 2^fix_bits
    double2* vol;
    double* w;
    double* pow;
    double* w2;
};

// Does particle P's plane come within reach of the tile for alias
// combination a (bit i set: axis i shifted by -N)?  Bitmask over the 8.
__device__ __forceinline__ unsigned tile_mask(const DevParticle& P, int x0, int y0, int z0, int N, int ft) {
    unsigned mask = 0;
    const float ex = 0.5f * (TX - 1), ey = 0.5f * (TY - 1), ez = 0.5f * (TZ - 1);
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

struct Tile {
    unsigned long long* re;
    unsigned long long* im;
    unsigned long long* w;
    unsigned long long* p;
    unsigned long long* q;
    float sF, sW, sP, sQ;      // fixed-point scales (powers of two)
};

template <bool FOM>
__device__ __forceinline__ void add_voxel(const Tile& T, int idx, float2 f, float w) {
    atomicAdd(T.re + idx, (unsigned long long)__float2ll_rn(f.x * w * T.sF));
    atomicAdd(T.im + idx, (unsigned long long)__float2ll_rn(f.y * w * T.sF));
    atomicAdd(T.w + idx, (unsigned long long)__float2ll_rn(w * T.sW));
    if (FOM) {
        atomicAdd(T.p + idx, (unsigned long long)__float2ll_rn(w * (f.x * f.x + f.y * f.y) * T.sP));
        atomicAdd(T.q + idx, (unsigned long long)__float2ll_rn(w * w * T.sQ));
    }
}

// Walk the pixels of one particle whose contributions reach the tile (alias
// origin ox, oy, oz): warp `warp` takes pixel rows k = k_lo + warp,
// + NWARPS, ...; lanes step along h.
template <bool FOM, bool GATE>
__device__ __forceinline__ void scatter_particle(const InsertArgs& a, const DevParticle& P, const float2* S,
                                                 const Tile& T, double ox, double oy, double oz, int warp,
                                                 int lane) {
    const int hf = a.ft / 2;
    // open box of map frequencies that touch the tile (tent support 1 voxel)
    const double lo[3] = {ox - 1.0, oy - 1.0, oz - 1.0};
    const double hi[3] = {ox + TX, oy + TY, oz + TZ};
    // pixel bounding box: the box projected on the plane's two axes
    double vc = 0, hv = 0, uc = 0, hu = 0;
    for (int i = 0; i < 3; ++i) {
        const double c = 0.5 * (lo[i] + hi[i]), e = 0.5 * (hi[i] - lo[i]);
        vc += P.bd[i] * c; hv += fabs(P.bd[i]) * e;
        uc += P.ad[i] * c; hu += fabs(P.ad[i]) * e;
    }
    vc *= P.inv_st2; hv *= P.inv_st2; uc *= P.inv_st2; hu *= P.inv_st2;
    const int k_lo = max((int)ceil(vc - hv), -hf), k_hi = min((int)floor(vc + hv), hf - 1);
    const int hb_lo = max((int)ceil(uc - hu), -hf), hb_hi = min((int)floor(uc + hu), hf - 1);
    const bool nearest = a.interp != 2;
    for (int k = k_lo + warp; k <= k_hi; k += NWARPS) {
        // h interval of row k: lo_i < h ad_i + k bd_i < hi_i on every axis
        double hl = hb_lo, hh = hb_hi;
        bool empty = false;
        for (int i = 0; i < 3; ++i) {
            const double base = k * P.bd[i];
            if (fabs(P.ad[i]) > 1e-12) {
                double p0 = (lo[i] - base) / P.ad[i], p1 = (hi[i] - base) / P.ad[i];
                if (p0 > p1) { const double t = p0; p0 = p1; p1 = t; }
                hl = fmax(hl, ceil(p0));
                hh = fmin(hh, floor(p1));
            } else if (!(base > lo[i] && base < hi[i])) {
                empty = true;
            }
        }
        if (empty || hl > hh) continue;
        const int h_lo = (int)hl, h_hi = (int)hh;
        const float2* row = S + (size_t)(k + hf) * a.pitch + hf;
        for (int h = h_lo + lane; h <= h_hi; h += 32) {
            float wt = P.pw;
            if (GATE) {
                bool keep;
                const float tw = pixel_weight_gate(a, P, h, k, keep);
                if (!keep) continue;
                wt *= tw;
            }
            const float2 f = __ldg(row + h);
            // map frequency relative to the tile origin, in double as the
            // reference forms it
            const double mx = h * P.ad[0] + k * P.bd[0] - ox;
            const double my = h * P.ad[1] + k * P.bd[1] - oy;
            const double mz = h * P.ad[2] + k * P.bd[2] - oz;
            if (nearest) {
                const double fx = floor(mx + 0.5), fy = floor(my + 0.5), fz = floor(mz + 0.5);
                const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
                if (ix < 0 || ix >= TX || iy < 0 || iy >= TY || iz < 0 || iz >= TZ) continue;
                float w = wt;
                if (a.interp == 1) {
                    const double dx = mx - fx, dy = my - fy, dz = mz - fz;
                    w = (float)((double)wt * (1.0 - sqrt(dx * dx + dy * dy + dz * dz)));
                }
                if (!(w > 0.f)) continue;
                add_voxel<FOM>(T, (iz * TY + iy) * TX + ix, f, w);
                continue;
            }
            const double flx = floor(mx), fly = floor(my), flz = floor(mz);
            const int ix = (int)flx, iy = (int)fly, iz = (int)flz;
            const float rx = (float)(mx - flx), ry = (float)(my - fly), rz = (float)(mz - flz);
            const float wx[2] = {1.f - rx, rx}, wy[2] = {1.f - ry, ry}, wz[2] = {1.f - rz, rz};
#pragma unroll
            for (int dz = 0; dz < 2; ++dz) {
                const int z = iz + dz;
                if (z < 0 || z >= TZ) continue;
#pragma unroll
                for (int dy = 0; dy < 2; ++dy) {
                    const int y = iy + dy;
                    if (y < 0 || y >= TY) continue;
                    const float wyz = wy[dy] * wz[dz] * wt;
#pragma unroll
                    for (int dx = 0; dx < 2; ++dx) {
                        const int x = ix + dx;
                        if (x < 0 || x >= TX) continue;
                        add_voxel<FOM>(T, (z * TY + y) * TX + x, f, wx[dx] * wyz);
                    }
                }
            }
        }
    }
}

__device__ __forceinline__ float pow2_scale(float maxval, int bits) {
    if (!(maxval > 0.f)) return 1.f;
    int e;
    frexpf(maxval, &e);                   // maxval < 2^e
    return ldexpf(1.f, bits - e);
}

template <bool FOM, bool GATE>
__global__ void __launch_bounds__(NT) insert_kernel(InsertArgs a) {
    const int N = a.N;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
    const int hf = a.ft / 2;
    const size_t spec_stride = (size_t)(2 * hf + 1) * a.pitch;

    extern __shared__ __align__(16) unsigned long long s_acc[];   // 3 or 5 channels x TV
    __shared__ unsigned s_list[NT];
    __shared__ int s_warp[NWARPS + 1];

    const int nch = FOM ? 5 : 3;
    for (int i = threadIdx.x; i < nch * TV; i += NT) s_acc[i] = 0ull;

    // fixed-point scales for this batch (identical in every block)
    const float fmax = __uint_as_float(*a.fmax_bits);
    Tile T;
    T.re = s_acc; T.im = s_acc + TV; T.w = s_acc + 2 * TV;
    T.p = FOM ? s_acc + 3 * TV : nullptr; T.q = FOM ? s_acc + 4 * TV : nullptr;
    T.sF = pow2_scale(fmax * a.pw_max, a.fix_bits);
    T.sW = pow2_scale(a.pw_max, a.fix_bits);
    T.sP = pow2_scale(fmax * fmax * 2.f * a.pw_max, a.fix_bits);
    T.sQ = pow2_scale(a.pw_max * a.pw_max, a.fix_bits);
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < a.np; base += NT) {
        const int p = base + threadIdx.x;
        unsigned mask = 0;
        if (p < a.np) {
            const DevParticle& P = a.part[p];
            if (P.half == a.half || a.half < 0) mask = tile_mask(P, x0, y0, z0, N, a.ft);
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
        const int cnt = s_warp[NWARPS];
        // every warp walks every listed particle (its own rows of each); the
        // integer sums make the order irrelevant, so warps never wait
        for (int e = 0; e < cnt; ++e) {
            const unsigned ent = s_list[e];
            const int pi = base + (int)(ent & 0xffffu);
            const DevParticle& P = a.part[pi];
            const float2* S = a.spec + (size_t)(a.p_base + pi) * spec_stride;
            for (int al = 0; al < 8; ++al) {
                if (!((ent >> (16 + al)) & 1u)) continue;
                scatter_particle<FOM, GATE>(a, P, S, T, (double)(x0 - ((al & 1) ? N : 0)),
                                            (double)(y0 - ((al & 2) ? N : 0)), (double)(z0 - ((al & 4) ? N : 0)),
                                            warp, lane);
            }
        }
        __syncthreads();
    }
    // fixed point -> double, added to the map accumulators
    const double iF = 1.0 / T.sF, iW = 1.0 / T.sW, iP = 1.0 / T.sP, iQ = 1.0 / T.sQ;
    for (int i = threadIdx.x; i < TV; i += NT) {
        const int lx = i % TX, ly = (i / TX) % TY, lz = i / (TX * TY);
        const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
        if (x >= N || y >= N || z >= N) continue;
        const size_t idx = ((size_t)z * N + y) * N + x;
        double2 o = a.vol[idx];
        o.x += (double)(long long)T.re[i] * iF;
        o.y += (double)(long long)T.im[i] * iF;
        a.vol[idx] = o;
        a.w[idx] += (double)(long long)T.w[i] * iW;
        if (FOM) {
            a.pow[idx] += (double)(long long)T.p[i] * iP;
            a.w2[idx] += (double)(long long)T.q[i] * iQ;
        }
    }
}

int tile_edge_for_step(double) { return 32; }

cudaError_t prepare_insert_attributes() {
    cudaError_t e = cudaFuncSetAttribute(insert_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(5 * TV * sizeof(unsigned long long)));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(insert_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(5 * TV * sizeof(unsigned long long)));
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
    a.fmax_bits = c.d_fmax;
    a.pw_max = c.pw_max;
    a.fix_bits = c.fix_bits;
    const int h = half < 0 ? 0 : half;
    a.vol = c.d_vol[h];
    a.w = c.d_w[h];
    a.pow = c.d_pow[h];
    a.w2 = c.d_w2[h];
    const int N = c.g.map;
    dim3 grid((N + TX - 1) / TX, (N + TY - 1) / TY, (N + TZ - 1) / TZ);
    const size_t smem = (c.g.fom ? 5 : 3) * TV * sizeof(unsigned long long);
    if (c.g.fom) {
        if (c.g.gate) insert_kernel<true, true><<<grid, NT, smem, s>>>(a);
        else insert_kernel<true, false><<<grid, NT, smem, s>>>(a);
    } else {
        if (c.g.gate) insert_kernel<false, true><<<grid, NT, smem, s>>>(a);
        else insert_kernel<false, false><<<grid, NT, smem, s>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace bsg
