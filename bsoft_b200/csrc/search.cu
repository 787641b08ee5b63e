// search.cu - exhaustive orientation search on sm_100a: every held particle
// image (at every trial origin) against a panel of central sections, scored
// by a BF16 correlation on the tensor cores (tcgen05, FP32 accumulators in
// TMEM), the best candidates of each image rescored with the exact FRC
// figure of merit of the reference (img_recip_space_fom).
//
// The reference refines locally (img_refine_grid, bsoft/src/mg/mg_refine.cpp:
// 1086-1195) and scores each hypothesis with img_recip_space_fom (:660-781):
//   FRC = (1/n_f) sum_j  sum_{p in j} Re(X_p conj(R_p) c_p)
//                        / sqrt(sum_{p in j} |X_p|^2  sum_{p in j} |R_p c_p|^2)
// over shells j < max_rad.  Written as one dot product per (image, section)
// pair it becomes a GEMM when the mixed term sum |R_p|^2 c_p^2 is split as
// (sum |R_p|^2) * mean_j(c_p^2), exact when the CTF is constant on a shell:
//   A[row = (image, origin)][p] = X_p e^{i phi_origin(p)} c_p / (n_f sqrt(D_j C_j))
//   B[col = section][p]         = R_p / sqrt(M_j)
// with D_j, C_j, M_j the shell sums of |X|^2, mean c^2, |R|^2 over the
// Hermitian half plane (the full-plane sums are twice these).  Complex
// products are real dot products of interleaved (re, im) pairs, so K = 2 x
// the half-plane pixels below max_rad, padded to 64.
//
// GEMM (C = A B^T, both K-major BF16): 128 x 256 output tiles, K-blocks of
// 64 staged by TMA (128-byte swizzle) through a 4-deep shared-memory ring;
// one elected thread issues tcgen05.mma (M=128, N=256, K=16) into one of two
// 256-column TMEM accumulators while four epilogue warps read the other with
// tcgen05.ld and keep each row's 8 best columns in registers.  Work items
// are (M tile, range of N tiles) so a CTA carries its rows' top-8 across the
// whole range; items are ordered so that the ~148 concurrent CTAs cover 10 M
// tiles x 15 N ranges and share their A and B tiles through L2.  Every wait
// is bounded (2 s) and reports through a status word.
#include "match.cuh"

#include <cuda.h>
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

namespace bsg {

namespace {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4, TOPK = 8;
constexpr int A_STAGE = BM * BK * 2;          // 16 KB
constexpr int B_STAGE = BN * BK * 2;          // 32 KB
constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
constexpr int GEMM_THREADS = 192;             // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int GEMM_SMEM = STAGES * STAGE_BYTES + 1024;
constexpr uint64_t WAIT_NS = 2000000000ull;   // bounded waits: 2 s

// instruction descriptor, kind::f16: D f32 (bits 4-5 = 1), A and B bf16
// (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t gtime() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// wait for the phase of `parity` to complete; false after WAIT_NS or when
// another role has given up
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = gtime();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 127) == 0) {
            if (*abort_flag) return false;
            if (gtime() - t0 > WAIT_NS) { *abort_flag = 1; return false; }
        }
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"((uint64_t)map), "r"(bar), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(IDESC), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row atoms
// 1024 bytes apart (SBO), version 1, base offset 0 (stage buffers are
// 1024-byte aligned)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

struct GemmArgs {
    int kblocks;          // K / 64
    int ncols;            // valid columns (sections)
    int ntiles_n;         // ceil(ncols / 256)
    int mtiles;           // M tiles holding rows of this batch
    long prow;            // row stride of the partial buffers (batch height)
    int ranges;           // N ranges
    int tiles_per_range;
    int mgroup;           // M tiles per group
    int items;            // groups * ranges * mgroup
    float* part_score;    // [ranges][prow][TOPK]
    int* part_idx;
    int* status;
};

__device__ __forceinline__ bool item_coords(const GemmArgs& a, int item, int& mtile, int& r) {
    const int per_group = a.ranges * a.mgroup;
    const int g = item / per_group, rem = item - g * per_group;
    r = rem / a.mgroup;
    mtile = g * a.mgroup + (rem - r * a.mgroup);
    return mtile < a.mtiles;
}

// keep the 8 largest (value, column) of a row, sorted descending
struct Top8 {
    float s[TOPK];
    int i[TOPK];
    __device__ __forceinline__ void reset() {
#pragma unroll
        for (int t = 0; t < TOPK; ++t) { s[t] = -3.0e38f; i[t] = -1; }
    }
    __device__ __forceinline__ void push(float v, int c) {
        if (!(v > s[TOPK - 1])) return;
        s[TOPK - 1] = v;
        i[TOPK - 1] = c;
#pragma unroll
        for (int t = TOPK - 1; t > 0; --t) {
            if (s[t] > s[t - 1]) {
                const float ts = s[t]; s[t] = s[t - 1]; s[t - 1] = ts;
                const int ti = i[t]; i[t] = i[t - 1]; i[t - 1] = ti;
            }
        }
    }
};

__global__ void __launch_bounds__(GEMM_THREADS, 1)
search_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs a) {
    extern __shared__ uint8_t gsm_raw[];
    __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], tfull_bar[2], tempty_bar[2], drain_bar;
    __shared__ uint32_t tmem_base_slot;
    __shared__ int abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t base = (smem_u32(gsm_raw) + 1023u) & ~1023u;   // 1024-aligned stage ring

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) { mbar_init(smem_u32(&full_bar[s]), 1); mbar_init(smem_u32(&empty_bar[s]), 1); }
        for (int s = 0; s < 2; ++s) { mbar_init(smem_u32(&tfull_bar[s]), 1); mbar_init(smem_u32(&tempty_bar[s]), 4); }
        mbar_init(smem_u32(&drain_bar), 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {   // TMEM: two 256-column fp32 accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                     "r"(512)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_slot;
    volatile int* abort_v = &abort_flag;

    if (warp == 0) {
        // ---- TMA producer ----
        if (lane == 0) {
            asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmA) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmB) : "memory");
            uint32_t stage = 0, phase = 0;
            uint32_t issued_mask = 0, last_parity = 0;   // per stage: ever issued, parity of its last load
            bool ok = true;
            for (int item = blockIdx.x; ok && item < a.items; item += gridDim.x) {
                int mtile, r;
                if (!item_coords(a, item, mtile, r)) continue;
                const int t0 = r * a.tiles_per_range, t1 = min(a.ntiles_n, t0 + a.tiles_per_range);
                for (int nt = t0; ok && nt < t1; ++nt) {
                    for (int kb = 0; kb < a.kblocks; ++kb) {
                        if (!mbar_wait(smem_u32(&empty_bar[stage]), phase ^ 1, abort_v)) { ok = false; break; }
                        const uint32_t fb = smem_u32(&full_bar[stage]);
                        mbar_expect_tx(fb, STAGE_BYTES);
                        const uint32_t sa = base + stage * STAGE_BYTES;
                        tma_load_2d(sa, &tmA, fb, kb * BK, mtile * BM);
                        tma_load_2d(sa + A_STAGE, &tmB, fb, kb * BK, nt * BN);
                        issued_mask |= 1u << stage;
                        last_parity = (last_parity & ~(1u << stage)) | (phase << stage);
                        if (++stage == STAGES) { stage = 0; phase ^= 1; }
                    }
                }
            }
            if (!ok) {
                // let the copies already issued land before the CTA can exit:
                // the phase of each stage's last load completes with its bytes
                for (int s = 0; s < STAGES; ++s) {
                    if (!(issued_mask >> s & 1)) continue;
                    const uint32_t par = (last_parity >> s) & 1;
                    const uint64_t t0 = gtime();
                    while (!mbar_try(smem_u32(&full_bar[s]), par) && gtime() - t0 < WAIT_NS) {
                    }
                }
                atomicOr(a.status, 1);
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer (one thread) ----
        if (lane == 0) {
            uint32_t stage = 0, phase = 0, acc = 0, aphase = 0;
            bool ok = true;
            for (int item = blockIdx.x; ok && item < a.items; item += gridDim.x) {
                int mtile, r;
                if (!item_coords(a, item, mtile, r)) continue;
                const int t0 = r * a.tiles_per_range, t1 = min(a.ntiles_n, t0 + a.tiles_per_range);
                for (int nt = t0; ok && nt < t1; ++nt) {
                    if (!mbar_wait(smem_u32(&tempty_bar[acc]), aphase ^ 1, abort_v)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t d = tmem + acc * BN;
                    for (int kb = 0; kb < a.kblocks; ++kb) {
                        if (!mbar_wait(smem_u32(&full_bar[stage]), phase, abort_v)) { ok = false; break; }
                        tc_fence_after();
                        const uint32_t sa = base + stage * STAGE_BYTES, sb = sa + A_STAGE;
#pragma unroll
                        for (int kk = 0; kk < BK / 16; ++kk)
                            tc_mma(d, sdesc(sa + kk * 32), sdesc(sb + kk * 32), (kb | kk) ? 1u : 0u);
                        tc_commit(smem_u32(&empty_bar[stage]));   // frees the stage when these MMAs finish
                        if (++stage == STAGES) { stage = 0; phase ^= 1; }
                    }
                    if (!ok) break;
                    tc_commit(smem_u32(&tfull_bar[acc]));         // accumulator ready
                    if (++acc == 2) { acc = 0; aphase ^= 1; }
                }
            }
            if (!ok) {
                // every MMA issued so far must finish before TMEM is released
                tc_commit(smem_u32(&drain_bar));
                const uint64_t t0 = gtime();
                while (!mbar_try(smem_u32(&drain_bar), 0) && gtime() - t0 < WAIT_NS) {
                }
                atomicOr(a.status, 2);
            }
        }
    } else {
        // ---- epilogue: warps 2..5, TMEM lane quarter = warp % 4 ----
        const int quarter = warp & 3;
        const uint32_t lane_off = (uint32_t)(quarter * 32) << 16;
        uint32_t acc = 0, aphase = 0;
        Top8 top;
        bool ok = true;
        for (int item = blockIdx.x; ok && item < a.items; item += gridDim.x) {
            int mtile, r;
            if (!item_coords(a, item, mtile, r)) continue;
            top.reset();
            const int t0 = r * a.tiles_per_range, t1 = min(a.ntiles_n, t0 + a.tiles_per_range);
            for (int nt = t0; nt < t1; ++nt) {
                // one lane waits, the warp follows it (tcgen05.ld is warp-collective)
                int w = 1;
                if (lane == 0) w = mbar_wait(smem_u32(&tfull_bar[acc]), aphase, abort_v) ? 1 : 0;
                w = __shfl_sync(0xffffffffu, w, 0);
                if (!w) { ok = false; break; }
                tc_fence_after();
                const uint32_t taddr = tmem + lane_off + acc * BN;
                for (int c = 0; c < BN; c += 32) {
                    uint32_t v[32];
                    tc_ld32(taddr + c, v);
                    const int col0 = nt * BN + c;
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (col0 + j < a.ncols) top.push(__uint_as_float(v[j]), col0 + j);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&tempty_bar[acc]));
                if (++acc == 2) { acc = 0; aphase ^= 1; }
            }
            if (!ok) break;
            const long row = (long)mtile * BM + quarter * 32 + lane;
            const long o = ((long)r * a.prow + row) * TOPK;
#pragma unroll
            for (int t = 0; t < TOPK; ++t) { a.part_score[o + t] = top.s[t]; a.part_idx[o + t] = top.i[t]; }
        }
        if (!ok && lane == 0) atomicOr(a.status, 4);
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
    }
}

// ---- panel and rows ---------------------------------------------------------

// one CTA per section: FSI-kernel gather of the coarse pixels (FP64
// accumulation), per-shell norms, BF16 row of interleaved (re, im)
__global__ void __launch_bounds__(256) panel_kernel(cudaTextureObject_t tex, int D,
                                                    const float* __restrict__ lut_g, int wd,
                                                    const MPix* __restrict__ cpix, int ncpix,
                                                    const int* __restrict__ cstart, int nf,
                                                    const MHyp* __restrict__ secs, double inv, double real, int kpad,
                                                    __nv_bfloat16* __restrict__ panel) {
    extern __shared__ float psm[];
    float* lut = psm;                                                // (NDIV+1)*MAXW
    float2* vals = reinterpret_cast<float2*>(psm + (NDIV + 1) * MAXW);   // ncpix
    float* gn = reinterpret_cast<float*>(vals + ncpix);              // nf
    for (int i = threadIdx.x; i < (NDIV + 1) * wd; i += blockDim.x) lut[i] = lut_g[i];
    __syncthreads();
    const MHyp& V = secs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int p = warp; p < ncpix; p += 8) {
        const MPix q = cpix[p];
        const double ix = q.h * inv, iy = q.k * inv;
        const double mx = (V.m[0] * ix + V.m[1] * iy) * real;
        const double my = (V.m[3] * ix + V.m[4] * iy) * real;
        const double mz = (V.m[6] * ix + V.m[7] * iy) * real;
        float vr, vi;
        fsi_gather<float>(TexSrc{tex}, D, mx, my, mz, lut, wd, lane, vr, vi);
        if (lane == 0) vals[p] = make_float2(vr, vi);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < nf; j += blockDim.x) {
        float m = 0.f;
        for (int p = cstart[j]; p < cstart[j + 1]; ++p) m += vals[p].x * vals[p].x + vals[p].y * vals[p].y;
        gn[j] = m > 0.f ? rsqrtf(m) : 0.f;
    }
    __syncthreads();
    __nv_bfloat162* row = reinterpret_cast<__nv_bfloat162*>(panel + (size_t)blockIdx.x * kpad);
    for (int p = threadIdx.x; p < kpad / 2; p += blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (p < ncpix) {
            const float g = gn[cpix[p].shell];
            v = make_float2(vals[p].x * g, vals[p].y * g);
        }
        row[p] = __floats2bfloat162_rn(v.x, v.y);
    }
}

// per image of the batch: 1 / (n_f sqrt(D_j C_j)) per coarse shell
__global__ void coarse_norm_kernel(const float2* __restrict__ spec, int D, const float* __restrict__ ctf, int npix,
                                   const MPix* __restrict__ cpix, const int* __restrict__ cstart, int nf, long img0,
                                   float* __restrict__ gA) {
    const long img = img0 + blockIdx.x;
    const float2* X = spec + img * (long)D * D;
    const float* C = ctf + img * (long)npix;
    for (int j = threadIdx.x; j < nf; j += blockDim.x) {
        double d = 0, c2 = 0;
        const int n = cstart[j + 1] - cstart[j];
        for (int p = cstart[j]; p < cstart[j + 1]; ++p) {
            const MPix q = cpix[p];
            const float2 x = X[q.idx];
            const double c = C[q.pad];
            d += (double)x.x * x.x + (double)x.y * x.y;
            c2 += c * c;
        }
        const double den = n > 0 ? d * (c2 / n) : 0.0;
        gA[(long)blockIdx.x * nf + j] = den > 0 ? (float)(1.0 / (nf * sqrt(den))) : 0.f;
    }
}

// one CTA per row (image, origin): X e^{i phi} c g as BF16 (re, im) pairs
__global__ void __launch_bounds__(256) rows_kernel(const float2* __restrict__ spec, int D, const float* __restrict__ ctf,
                                                   int npix, const MPix* __restrict__ cpix, int ncpix, int nf,
                                                   const float* __restrict__ gA, const double2* __restrict__ slopes,
                                                   int nshift, long img0, int kpad, __nv_bfloat16* __restrict__ A) {
    const int row = blockIdx.x;
    const int b = row / nshift, s = row - b * nshift;
    const long img = img0 + b;
    const float2* X = spec + img * (long)D * D;
    const float* C = ctf + img * (long)npix;
    const float* g = gA + (long)b * nf;
    const double2 sl = slopes[s];
    __nv_bfloat162* out = reinterpret_cast<__nv_bfloat162*>(A + (size_t)row * kpad);
    for (int p = threadIdx.x; p < kpad / 2; p += blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (p < ncpix) {
            const MPix q = cpix[p];
            const float2 x = X[q.idx];
            double phi = q.h * sl.x + q.k * sl.y;
            phi -= 6.283185307179586 * rint(phi * 0.15915494309189535);
            float sn, cs;
            sincosf((float)phi, &sn, &cs);
            const float f = C[q.pad] * g[q.shell];
            v = make_float2((x.x * cs - x.y * sn) * f, (x.x * sn + x.y * cs) * f);
        }
        out[p] = __floats2bfloat162_rn(v.x, v.y);
    }
}

// one warp per image: the topk best of its nshift rows x ranges x 8
// partial candidates (ties: lower section, then lower origin index)
__global__ void merge_kernel(const float* __restrict__ ps, const int* __restrict__ pi, int ranges, long mrows,
                             int nshift, int nimg_batch, int topk, long img0, int* __restrict__ cand_sec,
                             int* __restrict__ cand_org, float* __restrict__ cand_score) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= nimg_batch) return;
    const int n = nshift * ranges * TOPK;
    float prev_s = 3.0e38f;
    long prev_key = -1;
    for (int t = 0; t < topk; ++t) {
        float bs = -3.0e38f;
        long bk = -1;
        for (int e = lane; e < n; e += 32) {
            const int s = e / (ranges * TOPK), rem = e - s * ranges * TOPK, r = rem / TOPK, k = rem - r * TOPK;
            const long o = ((long)r * mrows + (long)warp * nshift + s) * TOPK + k;
            const int sec = pi[o];
            if (sec < 0) continue;
            const float v = ps[o];
            const long key = (long)sec * nshift + s;
            // strictly after the previous pick in (score desc, key asc) order
            const bool after = v < prev_s || (v == prev_s && key > prev_key);
            if (!after) continue;
            if (v > bs || (v == bs && (bk < 0 || key < bk))) { bs = v; bk = key; }
        }
        for (int o = 16; o; o >>= 1) {
            const float os = __shfl_xor_sync(0xffffffffu, bs, o);
            const long ok = __shfl_xor_sync(0xffffffffu, bk, o);
            if (ok >= 0 && (os > bs || (os == bs && (bk < 0 || ok < bk)))) { bs = os; bk = ok; }
        }
        if (lane == 0) {
            const long c = (img0 + warp) * topk + t;
            cand_sec[c] = bk >= 0 ? (int)(bk / nshift) : -1;
            cand_org[c] = bk >= 0 ? (int)(bk % nshift) : -1;
            cand_score[c] = bs;
        }
        prev_s = bs;
        prev_key = bk;
        if (bk < 0) prev_s = -3.0e38f;
    }
}


// ---- local search around proposals -----------------------------------------

constexpr int LOCAL_MAXC = 1024;    // candidate sections per image
constexpr int LOCAL_MAXO = 9;       // trial origins per image

// per image: the panel sections whose rotation lies within the angle whose
// cosine bound is `tr_min` of trace(R_p^T R_s) - in panel order (ordered
// compaction over 256-section chunks)
__global__ void __launch_bounds__(256) local_select_kernel(const float* __restrict__ prop, const float* __restrict__ rots,
                                                           long nsec, float tr_min, long img0,
                                                           int* __restrict__ cand, int* __restrict__ count) {
    __shared__ int wsum[8];
    __shared__ float Rp[9];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long img = img0 + blockIdx.x;
    if (threadIdx.x < 9) Rp[threadIdx.x] = prop[img * 11 + threadIdx.x];
    __syncthreads();
    int base_out = 0;
    int* my = cand + (long)blockIdx.x * LOCAL_MAXC;
    for (long c0 = 0; c0 < nsec; c0 += 256) {
        const long j = c0 + threadIdx.x;
        bool in = false;
        if (j < nsec) {
            const float* r = rots + j * 9;
            float t = 0.f;
#pragma unroll
            for (int k = 0; k < 9; ++k) t = fmaf(Rp[k], r[k], t);
            in = t >= tr_min;
        }
        const unsigned b = __ballot_sync(0xffffffffu, in);
        if (lane == 0) wsum[warp] = __popc(b);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < 8; ++w) { if (w < warp) before += wsum[w]; total += wsum[w]; }
        const int pos = base_out + before + __popc(b & ((1u << lane) - 1u));
        if (in && pos < LOCAL_MAXC) my[pos] = (int)j;
        base_out += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) count[blockIdx.x] = base_out;
}

__device__ __forceinline__ float2 bf2f(uint32_t u) {
    return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xFFFF0000u));
}

// per image: its A rows at its local origins in shared memory (BF16, as
// rows_kernel writes them), then every candidate section's panel row dotted
// with each of them by one warp; the topk (section, origin) pairs by score
// go to the candidate arrays in (score desc, section, origin) order
__global__ void __launch_bounds__(256) local_score_kernel(
    const float2* __restrict__ spec, int D, const float* __restrict__ ctf, int npix, const MPix* __restrict__ cpix,
    int ncpix, int nf, const float* __restrict__ gA, const double2* __restrict__ slopes,
    const int* __restrict__ lorg, const int* __restrict__ nlorg, const int* __restrict__ cand,
    const int* __restrict__ count, const __nv_bfloat16* __restrict__ panel, int kpad, int topk, long img0,
    int* __restrict__ out_sec, int* __restrict__ out_org, float* __restrict__ out_score) {
    extern __shared__ uint4 lsm[];
    const int b = blockIdx.x;
    const long img = img0 + b;
    const int no = nlorg[b];
    const int nc = min(count[b], LOCAL_MAXC);
    __nv_bfloat162* A = reinterpret_cast<__nv_bfloat162*>(lsm);           // no x kpad/2
    float* sc = reinterpret_cast<float*>(A + (size_t)LOCAL_MAXO * (kpad / 2));   // LOCAL_MAXC x LOCAL_MAXO
    const float2* X = spec + img * (long)D * D;
    const float* C = ctf + img * (long)npix;
    const float* g = gA + (long)b * nf;
    for (int o = 0; o < no; ++o) {
        const double2 sl = slopes[lorg[b * LOCAL_MAXO + o]];
        for (int p = threadIdx.x; p < kpad / 2; p += blockDim.x) {
            float2 v = make_float2(0.f, 0.f);
            if (p < ncpix) {
                const MPix q = cpix[p];
                const float2 x = X[q.idx];
                double phi = q.h * sl.x + q.k * sl.y;
                phi -= 6.283185307179586 * rint(phi * 0.15915494309189535);
                float sn, cs;
                sincosf((float)phi, &sn, &cs);
                const float f = C[q.pad] * g[q.shell];
                v = make_float2((x.x * cs - x.y * sn) * f, (x.x * sn + x.y * cs) * f);
            }
            A[(size_t)o * (kpad / 2) + p] = __floats2bfloat162_rn(v.x, v.y);
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint4* As = reinterpret_cast<const uint4*>(A);
    const int k8 = kpad / 8;                 // 16-byte chunks per row
    for (int ci = warp; ci < nc; ci += 8) {
        const int sec = cand[(long)b * LOCAL_MAXC + ci];
        const uint4* row = reinterpret_cast<const uint4*>(panel + (size_t)sec * kpad);
        float acc[LOCAL_MAXO];
#pragma unroll
        for (int o = 0; o < LOCAL_MAXO; ++o) acc[o] = 0.f;
        for (int p = lane; p < k8; p += 32) {
            const uint4 pb = __ldg(row + p);
            const float2 b0 = bf2f(pb.x), b1 = bf2f(pb.y), b2 = bf2f(pb.z), b3 = bf2f(pb.w);
#pragma unroll
            for (int o = 0; o < LOCAL_MAXO; ++o) {
                if (o < no) {
                    const uint4 ab = As[(size_t)o * k8 + p];
                    const float2 a0 = bf2f(ab.x), a1 = bf2f(ab.y), a2 = bf2f(ab.z), a3 = bf2f(ab.w);
                    float t = acc[o];
                    t = fmaf(a0.x, b0.x, t); t = fmaf(a0.y, b0.y, t);
                    t = fmaf(a1.x, b1.x, t); t = fmaf(a1.y, b1.y, t);
                    t = fmaf(a2.x, b2.x, t); t = fmaf(a2.y, b2.y, t);
                    t = fmaf(a3.x, b3.x, t); t = fmaf(a3.y, b3.y, t);
                    acc[o] = t;
                }
            }
        }
#pragma unroll
        for (int o = 0; o < LOCAL_MAXO; ++o) {
            float t = acc[o];
#pragma unroll
            for (int k = 16; k; k >>= 1) t += __shfl_xor_sync(0xffffffffu, t, k);
            if (lane == 0 && o < no) sc[ci * LOCAL_MAXO + o] = t;
        }
    }
    __syncthreads();
    if (warp == 0) {
        const int n = nc * no;
        float prev_s = 3.0e38f;
        long prev_k = -1;
        for (int t = 0; t < topk; ++t) {
            float bs = -3.0e38f;
            long bk = -1;
            for (int e = lane; e < n; e += 32) {
                const int ci = e / no, o = e - ci * no;
                const float v = sc[ci * LOCAL_MAXO + o];
                const long key = (long)cand[(long)b * LOCAL_MAXC + ci] * LOCAL_MAXO + o;
                const bool after = v < prev_s || (v == prev_s && key > prev_k);
                if (!after) continue;
                if (v > bs || (v == bs && (bk < 0 || key < bk))) { bs = v; bk = key; }
            }
            for (int k = 16; k; k >>= 1) {
                const float os = __shfl_xor_sync(0xffffffffu, bs, k);
                const long ok = __shfl_xor_sync(0xffffffffu, bk, k);
                if (ok >= 0 && (os > bs || (os == bs && (bk < 0 || ok < bk)))) { bs = os; bk = ok; }
            }
            if (lane == 0) {
                const long c = img * topk + t;
                out_sec[c] = bk >= 0 ? (int)(bk / LOCAL_MAXO) : -1;
                out_org[c] = bk >= 0 ? lorg[b * LOCAL_MAXO + (int)(bk % LOCAL_MAXO)] : -1;
                out_score[c] = bs;
            }
            prev_s = bk >= 0 ? bs : -3.0e38f;
            prev_k = bk;
        }
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// K-major BF16 matrix [rows][kpad] with a box of 64 x box_rows, 128B swizzle
bool make_map(CUtensorMap* m, const void* ptr, long rows, int kpad, int box_rows) {
    EncodeTiledFn f = encode_fn();
    if (!f) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)kpad, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)kpad * 2};
    const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

std::once_flag g_search_attr;
cudaError_t g_search_attr_err = cudaSuccess;

}  // namespace

// the coarse pixel list: half plane (k > 0, or k == 0 and h > 0), shells
// 1 .. n_f - 1, inside the section limit; .pad = index in the full list
static void coarse_pixels(Match& M) {
    M.h_cpix.clear();
    M.h_cstart.assign(M.nf + 1, 0);
    for (size_t i = 0; i < M.h_pix.size(); ++i) {
        MPix q = M.h_pix[i];
        if (q.shell < 1 || q.shell >= M.nf || !q.insec) continue;
        if (!(q.k > 0 || (q.k == 0 && q.h > 0))) continue;
        q.pad = (int)i;
        M.h_cpix.push_back(q);
        M.h_cstart[q.shell + 1]++;
    }
    for (int j = 0; j < M.nf; ++j) M.h_cstart[j + 1] += M.h_cstart[j];
    M.ncpix = (int)M.h_cpix.size();
    M.kpad = ((2 * M.ncpix + BK - 1) / BK) * BK;
}


// exact rescoring of the candidates in d_csec / d_corg / d_cscore (topk per
// held image): candidates of one image that share a section form one group
// (one gather, several origins); out gets each image's candidates ordered
// by the exact figure of merit
static cudaError_t rescore_candidates(Match& Mr, int topk, const std::vector<double2>& sl, double* out, float* tres,
                                      long* ngroups) {
    Match* M = &Mr;
    cudaStream_t s = M->stream;
    cudaError_t e = cudaSuccess;
    const long ncand = M->nimg * topk;
    std::vector<int> csec(ncand), corg(ncand);
    std::vector<float> cscore(ncand);
    e = cudaMemcpyAsync(csec.data(), M->d_csec, sizeof(int) * ncand, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(corg.data(), M->d_corg, sizeof(int) * ncand, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(cscore.data(), M->d_cscore, sizeof(float) * ncand, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    // groups of one image and one section (up to MAXORG origins), built per
    // image from the section index (the candidates of an image are adjacent)
    std::vector<MHypG> groups;
    std::vector<int> gsec;
    std::vector<long> cslot(ncand, -1);
    groups.reserve(ncand);
    for (long i = 0; i < M->nimg; ++i) {
        const size_t g0 = groups.size();
        for (int t = 0; t < topk; ++t) {
            const long c = i * topk + t;
            if (csec[c] < 0) continue;
            size_t g = groups.size();
            for (size_t q = g0; q < groups.size(); ++q)
                if (gsec[q] == csec[c] && groups[q].norg < MAXORG) { g = q; break; }
            if (g == groups.size()) {
                MHypG ng;
                memset(&ng, 0, sizeof(ng));
                memcpy(ng.m, M->h_secs[csec[c]].m, sizeof(ng.m));
                ng.img = (int)i;
                ng.ctf = (int)i;
                ng.sec = csec[c];          // row of the panel's exact sections
                groups.push_back(ng);
                gsec.push_back(csec[c]);
            }
            MHypG& G = groups[g];
            G.sx[G.norg] = sl[corg[c]].x;
            G.sy[G.norg] = sl[corg[c]].y;
            cslot[c] = (long)g * MAXORG + G.norg;
            G.norg++;
        }
    }
    const long ng = (long)groups.size();
    *ngroups = ng;
    std::vector<double> cf(2 * ncand, 0.0);
    *tres = 0;
    if (ng > 0) {
        if (ensure_groups(*M, ng) != BSG_OK) return cudaErrorMemoryAllocation;
        std::vector<double> go(2 * ng * MAXORG);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        e = cudaMemcpyAsync(M->d_grp, groups.data(), sizeof(MHypG) * ng, cudaMemcpyHostToDevice, s);
        cudaEventRecord(e0, s);
        if (e == cudaSuccess)
            e = launch_fom(*M, M->d_grp, ng, M->d_gout, M->d_gout + ng * MAXORG, s, false, nullptr, nullptr, false,
                           M->d_pexact);
        cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(go.data(), M->d_gout, sizeof(double) * go.size(), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaEventElapsedTime(tres, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (e != cudaSuccess) return e;
        for (long c = 0; c < ncand; ++c) {
            if (cslot[c] < 0) continue;
            cf[c] = go[cslot[c]];
            cf[ncand + c] = go[ng * MAXORG + cslot[c]];
        }
    }
    for (long i = 0; i < M->nimg; ++i) {
        std::vector<int> ord(topk);
        for (int t = 0; t < topk; ++t) ord[t] = t;
        const long b = i * topk;
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
            const bool vx = csec[b + x] >= 0, vy = csec[b + y] >= 0;
            if (vx != vy) return vx;
            return cf[b + x] > cf[b + y];
        });
        for (int t = 0; t < topk; ++t) {
            const long c = b + ord[t];
            double* o = out + (b + t) * BSG_MATCH_RESULT_DOUBLES;
            o[0] = csec[c];
            o[1] = corg[c];
            o[2] = cscore[c];
            o[3] = csec[c] >= 0 ? cf[c] : 0.0;
            o[4] = csec[c] >= 0 ? cf[ncand + c] : 0.0;
        }
    }
    return cudaSuccess;
}

}  // namespace bsg

using namespace bsg;

extern "C" int bsg_match_set_panel(bsg_match* h, const double* mats, long nsec, int flags) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !mats || nsec < 1) return match_fail(BSG_ERR_ARG, "bsg_match_set_panel: bad argument");
    if (!M->have_ref) return match_fail(BSG_ERR_STATE, "bsg_match_set_panel: set the reference first");
    cudaError_t e = cudaSetDevice(M->device);
    if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_set_panel: %s", cudaGetErrorString(e));
    std::call_once(g_search_attr, [] {
        g_search_attr_err = cudaFuncSetAttribute(search_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM);
        if (g_search_attr_err == cudaSuccess)
            g_search_attr_err = cudaFuncSetAttribute(panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    });
    if (g_search_attr_err != cudaSuccess)
        return match_fail(BSG_ERR_CUDA, "bsg_match_set_panel: %s", cudaGetErrorString(g_search_attr_err));
    coarse_pixels(*M);
    const size_t psmem = sizeof(float) * (NDIV + 1) * MAXW + sizeof(float2) * M->ncpix + sizeof(float) * M->nf;
    if (psmem > 200 * 1024) return match_fail(BSG_ERR_ARG, "bsg_match_set_panel: %d coarse pixels exceed the panel kernel's shared memory", M->ncpix);
    cudaStream_t s = M->stream;
    // release an older panel first
    cudaFree(M->d_panel); M->d_panel = nullptr;
    cudaFree(M->d_secs); M->d_secs = nullptr;
    cudaFree(M->d_cpix); M->d_cpix = nullptr;
    cudaFree(M->d_cstart); M->d_cstart = nullptr;
    cudaFree(M->d_rots); M->d_rots = nullptr;
    cudaFree(M->d_pexact); M->d_pexact = nullptr;
    M->nsec = 0;
    std::vector<MHyp> sv(nsec);
    for (long v = 0; v < nsec; ++v) {
        memset(&sv[v], 0, sizeof(MHyp));
        match_view_rows(*M, mats + 9 * v, sv[v].m);
    }
    e = cudaMalloc(&M->d_panel, sizeof(__nv_bfloat16) * (size_t)nsec * M->kpad);
    if (e == cudaSuccess) e = cudaMalloc(&M->d_secs, sizeof(MHyp) * nsec);
    if (e == cudaSuccess) e = cudaMalloc(&M->d_cpix, sizeof(MPix) * std::max(1, M->ncpix));
    if (e == cudaSuccess) e = cudaMalloc(&M->d_cstart, sizeof(int) * (M->nf + 1));
    if (e == cudaSuccess) e = cudaMalloc(&M->d_rots, sizeof(float) * 9 * nsec);
    if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_set_panel: %ld sections: %s", nsec, cudaGetErrorString(e));
    e = cudaMemcpyAsync(M->d_secs, sv.data(), sizeof(MHyp) * nsec, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(M->d_cpix, M->h_cpix.data(), sizeof(MPix) * M->ncpix, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(M->d_cstart, M->h_cstart.data(), sizeof(int) * (M->nf + 1), cudaMemcpyHostToDevice, s);
    {
        std::vector<float> rf((size_t)9 * nsec);
        for (long i = 0; i < 9 * nsec; ++i) rf[i] = (float)mats[i];
        if (e == cudaSuccess) e = cudaMemcpyAsync(M->d_rots, rf.data(), sizeof(float) * rf.size(), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    for (long v0 = 0; e == cudaSuccess && v0 < nsec; v0 += 1L << 20) {
        const long cnt = std::min(nsec - v0, 1L << 20);
        panel_kernel<<<(unsigned)cnt, 256, psmem, s>>>(M->ref_tex, M->D, M->d_lutf, M->wd, M->d_cpix, M->ncpix, M->d_cstart,
                                                       M->nf, M->d_secs + v0, 1.0 / M->real_map, M->real_map, M->kpad,
                                                       M->d_panel + (size_t)v0 * M->kpad);
        e = cudaGetLastError();
    }
    cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_set_panel: %s", cudaGetErrorString(e));
    M->nsec = nsec;
    M->h_secs.swap(sv);
    M->sstats.panel_ms += ms;
    M->sstats.launches += (nsec + (1L << 20) - 1) >> 20;
    // the panel's FP32 sections at the figure-of-merit pixels, kept for the
    // exact rescoring when they fit with 8 GB to spare (else the rescoring
    // gathers them per candidate)
    if (!(flags & BSG_MATCH_PANEL_GATHER)) {
        const size_t bytes = sizeof(float2) * (size_t)nsec * M->h_pix.size();
        size_t freeb = 0, total = 0;
        if (cudaMemGetInfo(&freeb, &total) == cudaSuccess && bytes + (8ull << 30) < freeb &&
            cudaMalloc(&M->d_pexact, bytes) == cudaSuccess) {
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            cudaEventRecord(e0, s);
            e = launch_panel_exact(*M, M->d_secs, nsec, M->d_pexact, s);
            cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            float xms = 0;
            cudaEventElapsedTime(&xms, e0, e1);
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            if (e != cudaSuccess) {
                cudaFree(M->d_pexact);
                M->d_pexact = nullptr;
                return match_fail(BSG_ERR_CUDA, "bsg_match_set_panel: exact sections: %s", cudaGetErrorString(e));
            }
            M->sstats.panel_exact_ms += xms;
            M->sstats.panel_exact_bytes = (double)bytes;
            M->sstats.launches += (nsec + (1L << 20) - 1) >> 20;
        } else {
            cudaGetLastError();     // a failed allocation leaves no sticky error; clear the last one
            M->sstats.panel_exact_bytes = 0;
        }
    }
    return BSG_OK;
}

extern "C" int bsg_match_search(bsg_match* h, const double* origins, int norigin, int topk, double* out, int flags) {
    (void)flags;
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !origins || !out || norigin < 1 || topk < 1 || topk > TOPK)
        return match_fail(BSG_ERR_ARG, "bsg_match_search: bad argument (topk must be 1..%d)", TOPK);
    if (M->nsec < 1 || M->nimg < 1) return match_fail(BSG_ERR_STATE, "bsg_match_search: set the panel and the images first");
    cudaError_t e = cudaSetDevice(M->device);
    if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_search: %s", cudaGetErrorString(e));
    cudaStream_t s = M->stream;
    const int nf = M->nf, kpad = M->kpad;
    // images per batch: rows of A (image x origin) up to ~256 MB
    const long row_bytes = 2L * kpad;
    long nb = std::max(1L, std::min<long>(M->nimg, (256L << 20) / (row_bytes * norigin)));
    if (M->cfg.batch > 0) nb = std::min<long>(nb, M->cfg.batch);
    const long rows_max = nb * norigin;
    const long mrows = ((rows_max + BM - 1) / BM) * BM;
    const int mtiles_max = (int)(mrows / BM);
    const int ntiles = (int)((M->nsec + BN - 1) / BN);
    // work-item grid: mgroup M tiles x ranges so that ~148 CTAs share tiles
    int mgroup = std::min(mtiles_max, 10);
    int ranges = std::max(1, std::min(ntiles, (148 + mgroup - 1) / mgroup));
    const int tpr = (ntiles + ranges - 1) / ranges;
    ranges = (ntiles + tpr - 1) / tpr;

    // scratch (kept between calls)
    const size_t need_A = (size_t)mrows * kpad;
    const size_t need_part = (size_t)ranges * mrows * TOPK;
    const size_t need_cand = (size_t)M->nimg * topk;
    if (need_A > M->a_elems) {
        cudaFree(M->d_A); M->d_A = nullptr; M->a_elems = 0;
        e = cudaMalloc(&M->d_A, sizeof(__nv_bfloat16) * need_A);
        if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_search: %s", cudaGetErrorString(e));
        M->a_elems = need_A;
    }
    if (need_part > M->part_elems) {
        cudaFree(M->d_pscore); cudaFree(M->d_pidx); M->d_pscore = nullptr; M->d_pidx = nullptr; M->part_elems = 0;
        e = cudaMalloc(&M->d_pscore, sizeof(float) * need_part);
        if (e == cudaSuccess) e = cudaMalloc(&M->d_pidx, sizeof(int) * need_part);
        if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_search: %s", cudaGetErrorString(e));
        M->part_elems = need_part;
    }
    if (need_cand > M->cand_elems) {
        cudaFree(M->d_csec); cudaFree(M->d_corg); cudaFree(M->d_cscore);
        M->d_csec = nullptr; M->d_corg = nullptr; M->d_cscore = nullptr;
        M->cand_elems = 0;
        e = cudaMalloc(&M->d_csec, sizeof(int) * need_cand);
        if (e == cudaSuccess) e = cudaMalloc(&M->d_corg, sizeof(int) * need_cand);
        if (e == cudaSuccess) e = cudaMalloc(&M->d_cscore, sizeof(float) * need_cand);
        if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_search: %s", cudaGetErrorString(e));
        M->cand_elems = need_cand;
    }
    if (M->gA_elems < (size_t)nb * nf) {
        cudaFree(M->d_gA); M->d_gA = nullptr;
        e = cudaMalloc(&M->d_gA, sizeof(float) * nb * nf);
        if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_search: %s", cudaGetErrorString(e));
        M->gA_elems = (size_t)nb * nf;
    }
    if (M->slope_elems < (size_t)norigin) {
        cudaFree(M->d_slopes); M->d_slopes = nullptr;
        e = cudaMalloc(&M->d_slopes, sizeof(double2) * norigin);
        if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_search: %s", cudaGetErrorString(e));
        M->slope_elems = norigin;
    }
    if (!M->d_status) {
        e = cudaMalloc(&M->d_status, sizeof(int));
        if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_search: %s", cudaGetErrorString(e));
    }
    // phase slopes of each trial origin (pixels of the uncut image, scaled
    // with the cut as change_transform_size does, then 2 pi o / diam)
    std::vector<double2> sl(norigin);
    for (int i = 0; i < norigin; ++i)
        sl[i] = make_double2(M->cut_scale * origins[2 * i] / M->D * 2 * M_PI, M->cut_scale * origins[2 * i + 1] / M->D * 2 * M_PI);
    e = cudaMemcpyAsync(M->d_slopes, sl.data(), sizeof(double2) * norigin, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(M->d_status, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(M->d_A, 0, sizeof(__nv_bfloat16) * need_A, s);
    if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_search: %s", cudaGetErrorString(e));

    CUtensorMap tmA, tmB;
    if (!make_map(&tmA, M->d_A, mrows, kpad, BM) || !make_map(&tmB, M->d_panel, M->nsec, kpad, BN))
        return match_fail(BSG_ERR_CUDA, "bsg_match_search: cuTensorMapEncodeTiled failed");

    cudaEvent_t ev[5];
    for (auto& x : ev) cudaEventCreate(&x);
    double agen = 0, gemm = 0, merge = 0;
    long launches = 0;
    for (long i0 = 0; e == cudaSuccess && i0 < M->nimg; i0 += nb) {
        const long cnt = std::min(nb, M->nimg - i0);
        const long rows = cnt * norigin;
        cudaEventRecord(ev[0], s);
        coarse_norm_kernel<<<(unsigned)cnt, 64, 0, s>>>(M->d_spec, M->D, M->d_ctf, (int)M->h_pix.size(), M->d_cpix,
                                                         M->d_cstart, nf, i0, M->d_gA);
        rows_kernel<<<(unsigned)rows, 256, 0, s>>>(M->d_spec, M->D, M->d_ctf, (int)M->h_pix.size(), M->d_cpix, M->ncpix,
                                                    nf, M->d_gA, M->d_slopes, norigin, i0, kpad, M->d_A);
        if (rows < mrows && i0 > 0)
            cudaMemsetAsync(M->d_A + (size_t)rows * kpad, 0, sizeof(__nv_bfloat16) * (mrows - rows) * kpad, s);
        cudaEventRecord(ev[1], s);
        GemmArgs ga{};
        ga.kblocks = kpad / BK;
        ga.ncols = (int)M->nsec;
        ga.ntiles_n = ntiles;
        ga.mtiles = (int)((rows + BM - 1) / BM);
        ga.prow = mrows;
        ga.mgroup = std::min(ga.mtiles, mgroup);
        ga.ranges = ranges;
        ga.tiles_per_range = tpr;
        const int groups = (ga.mtiles + ga.mgroup - 1) / ga.mgroup;
        ga.items = groups * ranges * ga.mgroup;
        ga.part_score = M->d_pscore;
        ga.part_idx = M->d_pidx;
        ga.status = M->d_status;
        const int grid = std::min(ga.items, 148);
        search_gemm_kernel<<<grid, GEMM_THREADS, GEMM_SMEM, s>>>(tmA, tmB, ga);
        cudaEventRecord(ev[2], s);
        merge_kernel<<<(unsigned)((cnt * 32 + 255) / 256), 256, 0, s>>>(M->d_pscore, M->d_pidx, ranges, mrows, norigin,
                                                                         (int)cnt, topk, i0, M->d_csec, M->d_corg,
                                                                         M->d_cscore);
        cudaEventRecord(ev[3], s);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[3]);
        float t01 = 0, t12 = 0, t23 = 0;
        cudaEventElapsedTime(&t01, ev[0], ev[1]);
        cudaEventElapsedTime(&t12, ev[1], ev[2]);
        cudaEventElapsedTime(&t23, ev[2], ev[3]);
        agen += t01;
        gemm += t12;
        merge += t23;
        launches += 4;
        int st = 0;
        if (e == cudaSuccess) e = cudaMemcpy(&st, M->d_status, sizeof(int), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && st) {
            for (auto& x : ev) cudaEventDestroy(x);
            return match_fail(BSG_ERR_CUDA, "bsg_match_search: the correlation kernel gave up waiting (status %d)", st);
        }
        M->sstats.gemm_flops += 2.0 * (double)rows * (double)M->nsec * (double)(2 * M->ncpix);
    }
    for (auto& x : ev) cudaEventDestroy(x);
    if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_search: %s", cudaGetErrorString(e));
    float tres = 0;
    long ng = 0;
    e = rescore_candidates(*M, topk, sl, out, &tres, &ng);
    if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_search: %s", cudaGetErrorString(e));
    const long ncand = M->nimg * topk;
    M->sstats.agen_ms += agen;
    M->sstats.gemm_ms += gemm;
    M->sstats.merge_ms += merge;
    M->sstats.rescore_ms += tres;
    M->sstats.launches += launches + (ng > 0 ? 1 : 0);
    M->sstats.gemm_launches += launches / 4;
    M->sstats.images += M->nimg;
    M->sstats.hypotheses += (double)M->nimg * norigin * (double)M->nsec;
    M->sstats.rescored += ncand;
    return BSG_OK;
}

extern "C" int bsg_match_get_stats(bsg_match* h, bsg_match_stats* st) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !st) return match_fail(BSG_ERR_ARG, "bsg_match_get_stats: null argument");
    *st = M->sstats;
    st->coarse_k = 2 * M->ncpix;
    st->kpad = M->kpad;
    return BSG_OK;
}

extern "C" int bsg_match_reset_stats(bsg_match* h) {
    Match* M = reinterpret_cast<Match*>(h);
    if (!M) return match_fail(BSG_ERR_ARG, "bsg_match_reset_stats: null argument");
    memset(&M->sstats, 0, sizeof(M->sstats));
    return BSG_OK;
}

extern "C" void* bsg_match_stream(bsg_match* h) {
    Match* M = reinterpret_cast<Match*>(h);
    return M ? static_cast<void*>(M->stream) : nullptr;
}

extern "C" int bsg_match_search_local(bsg_match* h, const float* proposals, double radius, const double* origins,
                                      int norigin, double origin_radius, int topk, double* out, int flags) {
    (void)flags;
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !proposals || !origins || !out || norigin < 1 || topk < 1 || topk > TOPK || !(radius > 0))
        return match_fail(BSG_ERR_ARG, "bsg_match_search_local: bad argument (topk must be 1..%d)", TOPK);
    if (M->nsec < 1 || M->nimg < 1) return match_fail(BSG_ERR_STATE, "bsg_match_search_local: set the panel and the images first");
    cudaError_t e = cudaSetDevice(M->device);
    if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_search_local: %s", cudaGetErrorString(e));
    static std::once_flag once;
    static cudaError_t attr = cudaSuccess;
    std::call_once(once, [] {
        attr = cudaFuncSetAttribute(local_score_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
    const size_t lsmem = sizeof(__nv_bfloat16) * (size_t)LOCAL_MAXO * M->kpad + sizeof(float) * LOCAL_MAXC * LOCAL_MAXO;
    if (attr != cudaSuccess || lsmem > 227 * 1024)
        return match_fail(BSG_ERR_ARG, "bsg_match_search_local: %d coarse values per row exceed the kernel's shared memory",
                          M->kpad);
    cudaStream_t s = M->stream;
    const long nimg = M->nimg;
    const int nf = M->nf;
    // local trial origins of each image: those within origin_radius of the
    // proposed origin (box centre + proposed shift), nearest first, at most 9
    std::vector<float> prop((size_t)nimg * 11);
    e = cudaMemcpy(prop.data(), proposals, sizeof(float) * prop.size(),
                   (flags & BSG_DEVICE_PTR) ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost);
    if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_search_local: %s", cudaGetErrorString(e));
    std::vector<int> lorg((size_t)nimg * LOCAL_MAXO, 0), nlorg(nimg, 0);
    for (long i = 0; i < nimg; ++i) {
        const double px = M->n / 2 + prop[i * 11 + 9], py = M->n / 2 + prop[i * 11 + 10];
        std::vector<std::pair<double, int>> d;
        for (int o = 0; o < norigin; ++o) {
            const double dx = origins[2 * o] - px, dy = origins[2 * o + 1] - py;
            d.push_back({dx * dx + dy * dy, o});
        }
        std::stable_sort(d.begin(), d.end());
        int k = 0;
        for (auto& t : d) {
            if (k >= LOCAL_MAXO || (t.first > origin_radius * origin_radius && k > 0)) break;
            lorg[i * LOCAL_MAXO + k++] = t.second;
        }
        nlorg[i] = k;
    }
    std::vector<double2> sl(norigin);
    for (int i = 0; i < norigin; ++i)
        sl[i] = make_double2(M->cut_scale * origins[2 * i] / M->D * 2 * M_PI, M->cut_scale * origins[2 * i + 1] / M->D * 2 * M_PI);
    const long nb = std::max(1L, std::min<long>(nimg, M->cfg.batch > 0 ? M->cfg.batch : 4096));
    // scratch
    const size_t need_cand = (size_t)nimg * topk;
    if (need_cand > M->cand_elems) {
        cudaFree(M->d_csec); cudaFree(M->d_corg); cudaFree(M->d_cscore);
        M->d_csec = nullptr; M->d_corg = nullptr; M->d_cscore = nullptr;
        M->cand_elems = 0;
        e = cudaMalloc(&M->d_csec, sizeof(int) * need_cand);
        if (e == cudaSuccess) e = cudaMalloc(&M->d_corg, sizeof(int) * need_cand);
        if (e == cudaSuccess) e = cudaMalloc(&M->d_cscore, sizeof(float) * need_cand);
        if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_search_local: %s", cudaGetErrorString(e));
        M->cand_elems = need_cand;
    }
    if (M->gA_elems < (size_t)nb * nf) {
        cudaFree(M->d_gA); M->d_gA = nullptr;
        e = cudaMalloc(&M->d_gA, sizeof(float) * nb * nf);
        if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_search_local: %s", cudaGetErrorString(e));
        M->gA_elems = (size_t)nb * nf;
    }
    if (M->slope_elems < (size_t)norigin) {
        cudaFree(M->d_slopes); M->d_slopes = nullptr;
        e = cudaMalloc(&M->d_slopes, sizeof(double2) * norigin);
        if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_search_local: %s", cudaGetErrorString(e));
        M->slope_elems = norigin;
    }
    // scratch kept in the context (grow-only): no allocation per call
    if (M->lscr_img < nimg) {
        cudaFree(M->d_lprop); cudaFree(M->d_lorg); cudaFree(M->d_nlorg);
        M->d_lprop = nullptr; M->d_lorg = nullptr; M->d_nlorg = nullptr;
        M->lscr_img = 0;
        e = cudaMalloc(&M->d_lprop, sizeof(float) * 11 * nimg);
        if (e == cudaSuccess) e = cudaMalloc(&M->d_lorg, sizeof(int) * LOCAL_MAXO * nimg);
        if (e == cudaSuccess) e = cudaMalloc(&M->d_nlorg, sizeof(int) * nimg);
        if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_search_local: %s", cudaGetErrorString(e));
        M->lscr_img = nimg;
    }
    if (M->lscr_nb < nb) {
        cudaFree(M->d_lcand); cudaFree(M->d_lcount);
        M->d_lcand = nullptr; M->d_lcount = nullptr;
        M->lscr_nb = 0;
        e = cudaMalloc(&M->d_lcand, sizeof(int) * nb * LOCAL_MAXC);
        if (e == cudaSuccess) e = cudaMalloc(&M->d_lcount, sizeof(int) * nb);
        if (e != cudaSuccess) return match_fail(BSG_ERR_NOMEM, "bsg_match_search_local: %s", cudaGetErrorString(e));
        M->lscr_nb = nb;
    }
    float* d_prop = M->d_lprop;
    int *d_lorg = M->d_lorg, *d_nlorg = M->d_nlorg, *d_cand = M->d_lcand, *d_count = M->d_lcount;
    e = cudaMemcpyAsync(d_prop, prop.data(), sizeof(float) * prop.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_lorg, lorg.data(), sizeof(int) * lorg.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_nlorg, nlorg.data(), sizeof(int) * nimg, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(M->d_slopes, sl.data(), sizeof(double2) * norigin, cudaMemcpyHostToDevice, s);
    const float tr_min = (float)(1.0 + 2.0 * cos(radius));
    cudaEvent_t ev[2];
    cudaEventCreate(&ev[0]);
    cudaEventCreate(&ev[1]);
    cudaEventRecord(ev[0], s);
    long launches = 0, considered = 0;
    std::vector<int> cnt_h(nb);
    for (long i0 = 0; e == cudaSuccess && i0 < nimg; i0 += nb) {
        const long cnt = std::min(nb, nimg - i0);
        local_select_kernel<<<(unsigned)cnt, 256, 0, s>>>(d_prop, M->d_rots, M->nsec, tr_min, i0, d_cand, d_count);
        coarse_norm_kernel<<<(unsigned)cnt, 64, 0, s>>>(M->d_spec, M->D, M->d_ctf, (int)M->h_pix.size(), M->d_cpix,
                                                         M->d_cstart, nf, i0, M->d_gA);
        local_score_kernel<<<(unsigned)cnt, 256, lsmem, s>>>(
            M->d_spec, M->D, M->d_ctf, (int)M->h_pix.size(), M->d_cpix, M->ncpix, nf, M->d_gA, M->d_slopes,
            d_lorg + i0 * LOCAL_MAXO, d_nlorg + i0, d_cand, d_count, M->d_panel, M->kpad, topk, i0, M->d_csec,
            M->d_corg, M->d_cscore);
        e = cudaGetLastError();
        launches += 3;
        if (e == cudaSuccess) e = cudaMemcpyAsync(cnt_h.data(), d_count, sizeof(int) * cnt, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        for (long i = 0; i < cnt; ++i) considered += (long)std::min(cnt_h[i], LOCAL_MAXC) * nlorg[i0 + i];
    }
    cudaEventRecord(ev[1], s);
    if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
    float lms = 0;
    cudaEventElapsedTime(&lms, ev[0], ev[1]);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_search_local: %s", cudaGetErrorString(e));
    float tres = 0;
    long ng = 0;
    e = rescore_candidates(*M, topk, sl, out, &tres, &ng);
    if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_search_local: %s", cudaGetErrorString(e));
    M->sstats.local_ms += lms;
    M->sstats.rescore_ms += tres;
    M->sstats.launches += launches + (ng > 0 ? 1 : 0);
    M->sstats.images += nimg;
    M->sstats.hypotheses += (double)considered;
    M->sstats.rescored += nimg * topk;
    return BSG_OK;
}
