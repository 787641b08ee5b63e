// cnn.cu - the learned orientation proposer: a small convolutional network
// that maps a particle image to a rotation (6-D representation, made
// orthonormal by Gram-Schmidt) and an in-plane shift, trained on the GPU by
// the kernels below.  It has no counterpart in the reference; it proposes
// poses for a local search whose scores are the reference's figure of merit.
//
// Network (activations NHWC, FP32; weights kept as FP32 masters and used
// rounded to BF16, products accumulated in FP32):
//   input  box x box x 1, normalised to zero mean and unit variance per image
//   6 x    3x3 convolution, stride 2, padding 1, bias, ReLU
//   fc1    (box/64)^2 * C6 -> hidden, ReLU
//   fc2    hidden -> 8 = a1(3), a2(3), shift(2)
//   head   b1 = a1/|a1|, b2 = normalised a2 - (b1.a2) b1, b3 = b1 x b2;
//          R = [b1 b2 b3] (columns), t = shift (pixels)
//   loss   mean over the batch of |R - R*|_F^2 + lambda |t - t*|^2
//
// Convolutions are GEMMs over im2col rows (M = batch x output pixels,
// K = 9 x input channels, N = output channels): forward C = X_col W^T,
// weight gradient W' = dY^T X_col (split over M, partial sums reduced in a
// fixed order), input gradient dX_col = dY W gathered back by col2im.  One
// tensor-core GEMM kernel (BF16 mma.sync with the operands split into two
// BF16 terms, FP32 accumulation, 128 x 64 tiles) serves all of them.  Every
// reduction has a fixed order, so training is bitwise reproducible for a
// given seed.
#include "common.cuh"

#include <cuda_bf16.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <random>
#include <vector>

namespace bsg {

namespace {

constexpr int NCONV = 6;
constexpr int NOUT = 8;     // a1, a2, shift
constexpr int NRES = 11;    // R (9, row-major) and shift (2)

// ---- GEMM: C[m][n] (+)= sum_k A(m, k) B(n, k) ------------------------------
// A(m, k) = AT ? A[k * lda + m] : A[m * lda + k]
// B(n, k) = BT ? B[k * ldb + n] : B[n * ldb + k]
// blockIdx.z splits k into `splits` ranges; with splits > 1 each range
// writes its own partial product C + z * M * N (reduced afterwards).
// On the tensor cores:
// mma.sync m16n8k16, BF16 operands, FP32 accumulation.  Every FP32 operand
// value v is split into hi = bf16(v) and lo = bf16(v - hi) while its tile is
// staged in shared memory, and each 16-deep step adds Ahi Bhi + Ahi Blo +
// Alo Bhi (the lo x lo term is below 2^-16 of the product), so a product
// keeps ~17 significant bits and the weights, which are BF16 values already,
// enter exactly (their lo parts are zero).  Block tile 128 x 64, eight warps
// of 32 x 32 (2 x 4 mma tiles); shared rows of 24 BF16 (12 words) so the
// fragment loads of the 8 row groups x 4 lanes fall on distinct banks.  The
// mma accumulation order is fixed, so results are bitwise reproducible.
constexpr int TBM = 128, TBN = 64, TBK = 16, TROW = 24;

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

template <bool AT, bool BT>
__global__ void __launch_bounds__(256) tgemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                    const float* __restrict__ B, int ldb, float* __restrict__ C,
                                                    int splits, int accumulate) {
    __shared__ __align__(16) __nv_bfloat16 Ah[TBM * TROW], Al[TBM * TROW], Bh[TBN * TROW], Bl[TBN * TROW];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = blockIdx.y * TBM, n0 = blockIdx.x * TBN;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int kper = (K + splits - 1) / splits;
    const int kb = blockIdx.z * kper, ke = min(K, kb + kper);
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;
    for (int k0 = kb; k0 < ke; k0 += TBK) {
        // A tile: TBM x TBK = 2048 values, 8 per thread
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int idx = tid + r * 256;
            int mm, kk;
            if (AT) { kk = idx / TBM; mm = idx % TBM; } else { mm = idx / TBK; kk = idx % TBK; }
            const int gm = m0 + mm, gk = k0 + kk;
            float v = 0.f;
            if (gm < M && gk < ke) v = AT ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
            split_bf16(v, Ah[mm * TROW + kk], Al[mm * TROW + kk]);
        }
        // B tile: TBN x TBK = 1024 values, 4 per thread
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int idx = tid + r * 256;
            int nn, kk;
            if (BT) { kk = idx / TBN; nn = idx % TBN; } else { nn = idx / TBK; kk = idx % TBK; }
            const int gn = n0 + nn, gk = k0 + kk;
            float v = 0.f;
            if (gn < N && gk < ke) v = BT ? B[(size_t)gk * ldb + gn] : B[(size_t)gn * ldb + gk];
            split_bf16(v, Bh[nn * TROW + kk], Bl[nn * TROW + kk]);
        }
        __syncthreads();
        uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int r0 = (wm + mt * 16 + g) * TROW, r8 = r0 + 8 * TROW;
            ah[mt][0] = *reinterpret_cast<const uint32_t*>(&Ah[r0 + 2 * t]);
            ah[mt][1] = *reinterpret_cast<const uint32_t*>(&Ah[r8 + 2 * t]);
            ah[mt][2] = *reinterpret_cast<const uint32_t*>(&Ah[r0 + 2 * t + 8]);
            ah[mt][3] = *reinterpret_cast<const uint32_t*>(&Ah[r8 + 2 * t + 8]);
            al[mt][0] = *reinterpret_cast<const uint32_t*>(&Al[r0 + 2 * t]);
            al[mt][1] = *reinterpret_cast<const uint32_t*>(&Al[r8 + 2 * t]);
            al[mt][2] = *reinterpret_cast<const uint32_t*>(&Al[r0 + 2 * t + 8]);
            al[mt][3] = *reinterpret_cast<const uint32_t*>(&Al[r8 + 2 * t + 8]);
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int c0 = (wn + nt * 8 + g) * TROW;
            bh[nt][0] = *reinterpret_cast<const uint32_t*>(&Bh[c0 + 2 * t]);
            bh[nt][1] = *reinterpret_cast<const uint32_t*>(&Bh[c0 + 2 * t + 8]);
            bl[nt][0] = *reinterpret_cast<const uint32_t*>(&Bl[c0 + 2 * t]);
            bl[nt][1] = *reinterpret_cast<const uint32_t*>(&Bl[c0 + 2 * t + 8]);
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                mma_bf16(acc[mt][nt], ah[mt], bh[nt]);
                mma_bf16(acc[mt][nt], ah[mt], bl[nt]);
                mma_bf16(acc[mt][nt], al[mt], bh[nt]);
            }
        __syncthreads();
    }
    float* Cz = C + (splits > 1 ? (size_t)blockIdx.z * M * N : 0);
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int gm = m0 + wm + mt * 16 + g + (q >= 2 ? 8 : 0);
                const int gn = n0 + wn + nt * 8 + 2 * t + (q & 1);
                if (gm >= M || gn >= N) continue;
                float* c = Cz + (size_t)gm * N + gn;
                *c = (accumulate && splits == 1) ? *c + acc[mt][nt][q] : acc[mt][nt][q];
            }
}

// sum of `splits` partial products into C (fixed order)
__global__ void split_reduce_kernel(const float* __restrict__ part, long count, int splits, float* __restrict__ C,
                                    int accumulate) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int z = 0; z < splits; ++z) s += part[(size_t)z * count + i];
        C[i] = accumulate ? C[i] + s : s;
    }
}

// ---- layers ------------------------------------------------------------------

// im2col for a 3x3, stride 2, padding 1 convolution over NHWC input:
// row (b, yo, xo), column (ky * 3 + kx) * Cin + ci
__global__ void im2col_kernel(const float* __restrict__ x, int B, int H, int W, int Cin, int Ho, int Wo,
                              float* __restrict__ col) {
    const long K = 9L * Cin, total = (long)B * Ho * Wo * K;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long row = i / K;
        const int kk = (int)(i - row * K);
        const int ci = kk % Cin, kyx = kk / Cin, ky = kyx / 3, kx = kyx % 3;
        const int xo = (int)(row % Wo), yo = (int)((row / Wo) % Ho), b = (int)(row / ((long)Wo * Ho));
        const int yi = 2 * yo + ky - 1, xi = 2 * xo + kx - 1;
        float v = 0.f;
        if (yi >= 0 && yi < H && xi >= 0 && xi < W) v = x[(((size_t)b * H + yi) * W + xi) * Cin + ci];
        col[i] = v;
    }
}

// input gradient: every input value gathers the column entries it fed
// (at most 2 x 2 taps for stride 2), in a fixed order
__global__ void col2im_kernel(const float* __restrict__ gcol, int B, int H, int W, int Cin, int Ho, int Wo,
                              float* __restrict__ gx) {
    const long total = (long)B * H * W * Cin;
    const long K = 9L * Cin;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int ci = (int)(i % Cin);
        const int xi = (int)((i / Cin) % W), yi = (int)((i / ((long)Cin * W)) % H), b = (int)(i / ((long)Cin * W * H));
        float s = 0.f;
        for (int ky = 0; ky < 3; ++ky) {
            const int t = yi + 1 - ky;
            if (t < 0 || (t & 1)) continue;
            const int yo = t >> 1;
            if (yo >= Ho) continue;
            for (int kx = 0; kx < 3; ++kx) {
                const int u = xi + 1 - kx;
                if (u < 0 || (u & 1)) continue;
                const int xo = u >> 1;
                if (xo >= Wo) continue;
                s += gcol[(((size_t)b * Ho + yo) * Wo + xo) * K + (ky * 3 + kx) * Cin + ci];
            }
        }
        gx[i] = s;
    }
}

// rows idx[b] of a (n x width) table
__global__ void gather_rows_kernel(const float* __restrict__ src, const int* __restrict__ idx, int rows, int width,
                                   float* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * width) return;
    const int r = i / width, c = i - r * width;
    dst[i] = src[(long)idx[r] * width + c];
}

__global__ void fill_kernel(float* __restrict__ p, long n, float v) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) p[i] = v;
}

// y[m][n] = relu?(y[m][n] + bias[n])
__global__ void bias_act_kernel(float* __restrict__ y, long M, int N, const float* __restrict__ bias, int relu) {
    const long total = M * N;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        float v = y[i] + bias[i % N];
        y[i] = relu ? fmaxf(v, 0.f) : v;
    }
}

// g *= (a > 0)
__global__ void relu_back_kernel(float* __restrict__ g, const float* __restrict__ a, long count) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x)
        if (!(a[i] > 0.f)) g[i] = 0.f;
}

// batch input: images idx[b] of the data set, normalised per image
// (population mean and standard deviation, FP64 sums in a fixed order)
__global__ void __launch_bounds__(256) gather_norm_kernel(const float* __restrict__ data, const int* __restrict__ idx,
                                                          int npix, float* __restrict__ out) {
    __shared__ double s1[256], s2[256];
    const long src = idx ? idx[blockIdx.x] : blockIdx.x;
    const float* p = data + src * (long)npix;
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < npix; i += 256) { const double v = p[i]; a += v; b += v * v; }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if (threadIdx.x < o) { s1[threadIdx.x] += s1[threadIdx.x + o]; s2[threadIdx.x] += s2[threadIdx.x + o]; }
        __syncthreads();
    }
    const double mean = s1[0] / npix;
    double var = s2[0] / npix - mean * mean;
    const float inv = var > 1e-30 ? (float)(1.0 / sqrt(var)) : 1.f;
    const float mu = (float)mean;
    float* q = out + (long)blockIdx.x * npix;
    for (int i = threadIdx.x; i < npix; i += 256) q[i] = (p[i] - mu) * inv;
}

__device__ __forceinline__ void cross3(const float* a, const float* b, float* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// head: outputs (B x 8) -> R (row-major, columns b1 b2 b3) and shift;
// with targets: per-sample loss and d loss / d outputs (mean over B)
__global__ void head_kernel(const float* __restrict__ o, int B, const float* __restrict__ tgt, float lambda,
                            float* __restrict__ res, float* __restrict__ go, float* __restrict__ loss) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const float* a1 = o + b * NOUT;
    const float* a2 = a1 + 3;
    const float n1 = sqrtf(a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2]) + 1e-12f;
    float b1[3] = {a1[0] / n1, a1[1] / n1, a1[2] / n1};
    const float d = b1[0] * a2[0] + b1[1] * a2[1] + b1[2] * a2[2];
    float u2[3] = {a2[0] - d * b1[0], a2[1] - d * b1[1], a2[2] - d * b1[2]};
    const float n2 = sqrtf(u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]) + 1e-12f;
    float b2[3] = {u2[0] / n2, u2[1] / n2, u2[2] / n2};
    float b3[3];
    cross3(b1, b2, b3);
    const float t0 = o[b * NOUT + 6], t1 = o[b * NOUT + 7];
    if (res) {
        float* r = res + b * NRES;
        for (int i = 0; i < 3; ++i) { r[3 * i + 0] = b1[i]; r[3 * i + 1] = b2[i]; r[3 * i + 2] = b3[i]; }
        r[9] = t0;
        r[10] = t1;
    }
    if (!tgt) return;
    const float* T = tgt + b * NRES;    // R* row-major, t*
    float r1[3] = {T[0], T[3], T[6]}, r2[3] = {T[1], T[4], T[7]}, r3[3] = {T[2], T[5], T[8]};
    float L = 0.f, gb1[3], gb2[3], gb3[3];
    for (int i = 0; i < 3; ++i) {
        gb1[i] = 2.f * (b1[i] - r1[i]);
        gb2[i] = 2.f * (b2[i] - r2[i]);
        gb3[i] = 2.f * (b3[i] - r3[i]);
        L += (b1[i] - r1[i]) * (b1[i] - r1[i]) + (b2[i] - r2[i]) * (b2[i] - r2[i]) + (b3[i] - r3[i]) * (b3[i] - r3[i]);
    }
    const float dt0 = t0 - T[9], dt1 = t1 - T[10];
    L += lambda * (dt0 * dt0 + dt1 * dt1);
    // b3 = b1 x b2: d/db1 (g.b3) = b2 x g, d/db2 (g.b3) = g x b1
    float c[3];
    cross3(b2, gb3, c);
    for (int i = 0; i < 3; ++i) gb1[i] += c[i];
    cross3(gb3, b1, c);
    for (int i = 0; i < 3; ++i) gb2[i] += c[i];
    // b2 = u2 / n2
    const float gb2b2 = gb2[0] * b2[0] + gb2[1] * b2[1] + gb2[2] * b2[2];
    float gu2[3];
    for (int i = 0; i < 3; ++i) gu2[i] = (gb2[i] - gb2b2 * b2[i]) / n2;
    // u2 = a2 - (b1.a2) b1
    const float gu2b1 = gu2[0] * b1[0] + gu2[1] * b1[1] + gu2[2] * b1[2];
    float ga2[3];
    for (int i = 0; i < 3; ++i) {
        ga2[i] = gu2[i] - gu2b1 * b1[i];
        gb1[i] += -d * gu2[i] - a2[i] * gu2b1;
    }
    // b1 = a1 / n1
    const float gb1b1 = gb1[0] * b1[0] + gb1[1] * b1[1] + gb1[2] * b1[2];
    const float sc = 1.f / B;
    float* g = go + b * NOUT;
    for (int i = 0; i < 3; ++i) {
        g[i] = sc * (gb1[i] - gb1b1 * b1[i]) / n1;
        g[3 + i] = sc * ga2[i];
    }
    g[6] = sc * 2.f * lambda * dt0;
    g[7] = sc * 2.f * lambda * dt1;
    loss[b] = L;
}

__global__ void mean_kernel(const float* __restrict__ v, int n, float* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0;
        for (int i = 0; i < n; ++i) s += v[i];
        *out = (float)(s / n);
    }
}

// Adam on the FP32 masters; the working copy is the BF16 rounding
__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ weff, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, long n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        w[i] = wi;
        weff[i] = __bfloat162float(__float2bfloat16_rn(wi));
    }
}

__global__ void round_bf16_kernel(const float* __restrict__ w, float* __restrict__ weff, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        weff[i] = __bfloat162float(__float2bfloat16_rn(w[i]));
}

struct Layer {
    int cin, cout, h, w, ho, wo;   // convolution geometry (fc: h = w = ho = wo = 1)
    long woff, boff, k;            // weight / bias offsets, K = 9 cin (conv) or cin (fc)
};

}  // namespace

struct Cnn {
    bsg_cnn_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    Layer conv[NCONV], fc1, fc2;
    long nparams = 0;
    float *d_w = nullptr, *d_weff = nullptr, *d_g = nullptr, *d_m = nullptr, *d_v = nullptr;
    int cap = 0;                       // batch capacity of the buffers
    float* d_in = nullptr;             // cap x box^2
    float* d_act[NCONV + 1] = {};      // NHWC activations after ReLU (act[0] = input)
    float* d_h = nullptr;              // fc1 output
    float* d_o = nullptr;              // fc2 output
    float* d_col = nullptr;            // im2col scratch
    float* d_gcol = nullptr;
    float* d_ga = nullptr;             // activation gradient scratch (two halves)
    float* d_gb = nullptr;
    float* d_gh = nullptr;
    float* d_go = nullptr;
    float* d_part = nullptr;           // split-K partials
    float* d_ones = nullptr;           // column sums as a GEMM with a ones row
    long ones_elems = 0;
    size_t part_elems = 0;
    float* d_res = nullptr;            // cap x 11
    float* d_tgt = nullptr;            // cap x 11
    float* d_loss = nullptr;           // cap
    float* d_lossmean = nullptr;       // per step
    int* d_idx = nullptr;
    long step = 0;                     // Adam steps taken
    size_t col_elems = 0, act_max = 0;
};

}  // namespace bsg

using namespace bsg;

namespace {

int cfail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_error("%s", buf);
    return code;
}

#define CCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return cfail(BSG_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

unsigned grid_for(long n) { return (unsigned)std::max(1L, std::min(148L * 16, (n + 255) / 256)); }

cudaError_t gemm(Cnn& c, bool at, bool bt, int M, int N, int K, const float* A, int lda, const float* B, int ldb,
                 float* C, int accumulate, cudaStream_t s);

// column sums of g (M x N), as ones(1 x M) g: fixed-order split reduction
cudaError_t colsum(Cnn& c, const float* g, long M, int N, float* out, cudaStream_t s) {
    return gemm(c, false, true, 1, N, (int)M, c.d_ones, (int)M, g, N, out, 0, s);
}

cudaError_t gemm(Cnn& c, bool at, bool bt, int M, int N, int K, const float* A, int lda, const float* B, int ldb,
                 float* C, int accumulate, cudaStream_t s) {
    dim3 grid((N + TBN - 1) / TBN, (M + TBM - 1) / TBM, 1);
    int splits = 1;
    const long tiles = (long)grid.x * grid.y;
    if (tiles < 148 && K > 4096) {
        splits = (int)std::min<long>(64, std::max<long>(1, (296 + tiles - 1) / tiles));
        splits = std::min(splits, std::max(1, K / 1024));
        if ((size_t)splits * M * N > c.part_elems) splits = std::max(1, (int)(c.part_elems / ((size_t)M * N)));
    }
    grid.z = splits;
    float* out = splits > 1 ? c.d_part : C;
    if (!at && !bt) tgemm_kernel<false, false><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, out, splits, accumulate);
    else if (!at && bt) tgemm_kernel<false, true><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, out, splits, accumulate);
    else if (at && !bt) tgemm_kernel<true, false><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, out, splits, accumulate);
    else tgemm_kernel<true, true><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, out, splits, accumulate);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && splits > 1) {
        const long cnt = (long)M * N;
        split_reduce_kernel<<<grid_for(cnt), 256, 0, s>>>(c.d_part, cnt, splits, C, accumulate);
        e = cudaGetLastError();
    }
    return e;
}

int ensure_batch(Cnn& c, int B) {
    if (B <= c.cap) return BSG_OK;
    auto F = [](float*& p) { cudaFree(p); p = nullptr; };
    F(c.d_in); for (auto& a : c.d_act) F(a);
    F(c.d_h); F(c.d_o); F(c.d_col); F(c.d_gcol); F(c.d_ga); F(c.d_gb); F(c.d_gh); F(c.d_go); F(c.d_part);
    F(c.d_res); F(c.d_tgt); F(c.d_loss); F(c.d_ones);
    cudaFree(c.d_idx); c.d_idx = nullptr;
    const int box = c.cfg.box;
    size_t col = 0, act = (size_t)box * box;
    for (int l = 0; l < NCONV; ++l) {
        const Layer& L = c.conv[l];
        col = std::max(col, (size_t)L.ho * L.wo * L.k);
        act = std::max(act, (size_t)L.ho * L.wo * L.cout);
    }
    c.col_elems = col * B;
    c.act_max = act * B;
    CCK(cudaMalloc(&c.d_in, sizeof(float) * (size_t)box * box * B));
    c.d_act[0] = c.d_in;
    for (int l = 0; l < NCONV; ++l) {
        const Layer& L = c.conv[l];
        CCK(cudaMalloc(&c.d_act[l + 1], sizeof(float) * (size_t)L.ho * L.wo * L.cout * B));
    }
    CCK(cudaMalloc(&c.d_h, sizeof(float) * (size_t)c.cfg.hidden * B));
    CCK(cudaMalloc(&c.d_o, sizeof(float) * NOUT * B));
    CCK(cudaMalloc(&c.d_col, sizeof(float) * c.col_elems));
    CCK(cudaMalloc(&c.d_gcol, sizeof(float) * c.col_elems));
    CCK(cudaMalloc(&c.d_ga, sizeof(float) * c.act_max));
    CCK(cudaMalloc(&c.d_gb, sizeof(float) * c.act_max));
    CCK(cudaMalloc(&c.d_gh, sizeof(float) * (size_t)c.cfg.hidden * B));
    CCK(cudaMalloc(&c.d_go, sizeof(float) * NOUT * B));
    c.part_elems = std::max<size_t>((size_t)1 << 22, (size_t)c.cfg.hidden * 1024 * 4);
    CCK(cudaMalloc(&c.d_part, sizeof(float) * c.part_elems));
    CCK(cudaMalloc(&c.d_res, sizeof(float) * NRES * B));
    CCK(cudaMalloc(&c.d_tgt, sizeof(float) * NRES * B));
    CCK(cudaMalloc(&c.d_loss, sizeof(float) * B));
    CCK(cudaMalloc(&c.d_idx, sizeof(int) * B));
    c.ones_elems = (long)B * (box / 2) * (box / 2);
    CCK(cudaMalloc(&c.d_ones, sizeof(float) * c.ones_elems));
    fill_kernel<<<grid_for(c.ones_elems), 256>>>(c.d_ones, c.ones_elems, 1.f);
    CCK(cudaGetLastError());
    CCK(cudaDeviceSynchronize());
    c.cap = B;
    return BSG_OK;
}

// forward pass of B images already in c.d_in (normalised)
cudaError_t forward(Cnn& c, int B, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    for (int l = 0; l < NCONV && e == cudaSuccess; ++l) {
        const Layer& L = c.conv[l];
        const long M = (long)B * L.ho * L.wo;
        im2col_kernel<<<grid_for(M * L.k), 256, 0, s>>>(c.d_act[l], B, L.h, L.w, L.cin, L.ho, L.wo, c.d_col);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = gemm(c, false, false, (int)M, L.cout, (int)L.k, c.d_col, (int)L.k, c.d_weff + L.woff, (int)L.k,
                     c.d_act[l + 1], 0, s);
        if (e == cudaSuccess) {
            bias_act_kernel<<<grid_for(M * L.cout), 256, 0, s>>>(c.d_act[l + 1], M, L.cout, c.d_weff + L.boff, 1);
            e = cudaGetLastError();
        }
    }
    const Layer& F1 = c.fc1;
    const Layer& F2 = c.fc2;
    if (e == cudaSuccess)
        e = gemm(c, false, false, B, F1.cout, (int)F1.k, c.d_act[NCONV], (int)F1.k, c.d_weff + F1.woff, (int)F1.k, c.d_h,
                 0, s);
    if (e == cudaSuccess) {
        bias_act_kernel<<<grid_for((long)B * F1.cout), 256, 0, s>>>(c.d_h, B, F1.cout, c.d_weff + F1.boff, 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = gemm(c, false, false, B, F2.cout, (int)F2.k, c.d_h, (int)F2.k, c.d_weff + F2.woff, (int)F2.k, c.d_o, 0, s);
    if (e == cudaSuccess) {
        bias_act_kernel<<<grid_for((long)B * F2.cout), 256, 0, s>>>(c.d_o, B, F2.cout, c.d_weff + F2.boff, 0);
        e = cudaGetLastError();
    }
    return e;
}

// gradients of the batch loss into c.d_g (overwritten), from c.d_go
cudaError_t backward(Cnn& c, int B, cudaStream_t s) {
    const Layer& F1 = c.fc1;
    const Layer& F2 = c.fc2;
    const int H = c.cfg.hidden;
    // fc2: dW2 = go^T h, db2 = sum go, dh = go W2
    cudaError_t e = gemm(c, true, true, F2.cout, H, B, c.d_go, NOUT, c.d_h, H, c.d_g + F2.woff, 0, s);
    if (e == cudaSuccess) e = colsum(c, c.d_go, B, NOUT, c.d_g + F2.boff, s);
    if (e == cudaSuccess) e = gemm(c, false, true, B, H, NOUT, c.d_go, NOUT, c.d_weff + F2.woff, H, c.d_gh, 0, s);
    if (e == cudaSuccess) { relu_back_kernel<<<grid_for((long)B * H), 256, 0, s>>>(c.d_gh, c.d_h, (long)B * H); e = cudaGetLastError(); }
    // fc1: dW1 = gh^T a6, db1, da6 = gh W1
    const int K1 = (int)F1.k;
    if (e == cudaSuccess) e = gemm(c, true, true, H, K1, B, c.d_gh, H, c.d_act[NCONV], K1, c.d_g + F1.woff, 0, s);
    if (e == cudaSuccess) e = colsum(c, c.d_gh, B, H, c.d_g + F1.boff, s);
    float* ga = c.d_ga;   // gradient w.r.t. act[l+1]
    float* gb = c.d_gb;
    if (e == cudaSuccess) e = gemm(c, false, true, B, K1, H, c.d_gh, H, c.d_weff + F1.woff, K1, ga, 0, s);
    for (int l = NCONV - 1; l >= 0 && e == cudaSuccess; --l) {
        const Layer& L = c.conv[l];
        const long M = (long)B * L.ho * L.wo;
        relu_back_kernel<<<grid_for(M * L.cout), 256, 0, s>>>(ga, c.d_act[l + 1], M * L.cout);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = colsum(c, ga, M, L.cout, c.d_g + L.boff, s);
        if (e == cudaSuccess) {
            im2col_kernel<<<grid_for(M * L.k), 256, 0, s>>>(c.d_act[l], B, L.h, L.w, L.cin, L.ho, L.wo, c.d_col);
            e = cudaGetLastError();
        }
        // dW = dY^T X_col  (Cout x K, reduced over M)
        if (e == cudaSuccess)
            e = gemm(c, true, true, L.cout, (int)L.k, (int)M, ga, L.cout, c.d_col, (int)L.k, c.d_g + L.woff, 0, s);
        if (l > 0 && e == cudaSuccess) {
            // dX_col = dY W  (M x K), then col2im into the previous activation's gradient
            e = gemm(c, false, true, (int)M, (int)L.k, L.cout, ga, L.cout, c.d_weff + L.woff, (int)L.k, c.d_gcol, 0, s);
            if (e == cudaSuccess) {
                const long nx = (long)B * L.h * L.w * L.cin;
                col2im_kernel<<<grid_for(nx), 256, 0, s>>>(c.d_gcol, B, L.h, L.w, L.cin, L.ho, L.wo, gb);
                e = cudaGetLastError();
            }
            std::swap(ga, gb);
        }
    }
    return e;
}

uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

extern "C" int bsg_cnn_create(const bsg_cnn_config* cfg, bsg_cnn** out) {
    if (!cfg || !out) return cfail(BSG_ERR_ARG, "bsg_cnn_create: null argument");
    *out = nullptr;
    const int box = cfg->box;
    if (box < 64 || box > 512 || (box & (box - 1)))
        return cfail(BSG_ERR_ARG, "bsg_cnn_create: box %d must be a power of two in 64..512", box);
    for (int l = 0; l < NCONV; ++l)
        if (cfg->channels[l] < 1 || cfg->channels[l] > 1024) return cfail(BSG_ERR_ARG, "bsg_cnn_create: bad channel count");
    if (cfg->hidden < 1 || cfg->hidden > 8192) return cfail(BSG_ERR_ARG, "bsg_cnn_create: bad hidden width");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev)
        return cfail(BSG_ERR_NODEV, "bsg_cnn_create: no CUDA device %d", cfg->device);
    CCK(cudaSetDevice(cfg->device));
    Cnn* c = new (std::nothrow) Cnn();
    if (!c) return cfail(BSG_ERR_NOMEM, "bsg_cnn_create: out of host memory");
    c->cfg = *cfg;
    c->device = cfg->device;
    long off = 0;
    int h = box, cin = 1;
    for (int l = 0; l < NCONV; ++l) {
        Layer& L = c->conv[l];
        L.cin = cin; L.cout = cfg->channels[l]; L.h = L.w = h; L.ho = L.wo = h / 2; L.k = 9L * cin;
        L.woff = off; off += (long)L.cout * L.k;
        L.boff = off; off += L.cout;
        cin = L.cout;
        h /= 2;
    }
    c->fc1 = Layer{h * h * cin, cfg->hidden, 1, 1, 1, 1, off, 0, (long)h * h * cin};
    off += (long)c->fc1.cout * c->fc1.k;
    c->fc1.boff = off; off += c->fc1.cout;
    c->fc2 = Layer{cfg->hidden, NOUT, 1, 1, 1, 1, off, 0, cfg->hidden};
    off += (long)NOUT * cfg->hidden;
    c->fc2.boff = off; off += NOUT;
    c->nparams = off;
    // He initialisation from a seeded generator; biases zero
    std::vector<float> w(off, 0.f);
    uint64_t st = cfg->seed ? cfg->seed : 0x5EEDull;
    auto normal = [&]() {
        const double u1 = ((splitmix(st) >> 11) + 1.0) / 9007199254740993.0, u2 = (splitmix(st) >> 11) / 9007199254740992.0;
        return sqrt(-2.0 * log(u1)) * cos(2 * M_PI * u2);
    };
    auto init = [&](const Layer& L) {
        const double sd = sqrt(2.0 / L.k);
        for (long i = 0; i < (long)L.cout * L.k; ++i) w[L.woff + i] = (float)(sd * normal());
    };
    for (int l = 0; l < NCONV; ++l) init(c->conv[l]);
    init(c->fc1);
    {
        const double sd = sqrt(1.0 / c->fc2.k);
        for (long i = 0; i < (long)NOUT * c->fc2.k; ++i) w[c->fc2.woff + i] = (float)(sd * normal());
    }
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_w, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_weff, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_g, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_m, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_v, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_lossmean, sizeof(float) * 1);
    if (e == cudaSuccess) e = cudaMemcpy(c->d_w, w.data(), sizeof(float) * off, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(c->d_m, 0, sizeof(float) * off);
    if (e == cudaSuccess) e = cudaMemset(c->d_v, 0, sizeof(float) * off);
    if (e == cudaSuccess) {
        round_bf16_kernel<<<grid_for(off), 256, 0, c->stream>>>(c->d_w, c->d_weff, off);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        bsg_cnn_destroy(reinterpret_cast<bsg_cnn*>(c));
        return cfail(BSG_ERR_CUDA, "bsg_cnn_create: %s", cudaGetErrorString(e));
    }
    *out = reinterpret_cast<bsg_cnn*>(c);
    return BSG_OK;
}

extern "C" void bsg_cnn_destroy(bsg_cnn* h) {
    Cnn* c = reinterpret_cast<Cnn*>(h);
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    float* fp[] = {c->d_w, c->d_weff, c->d_g, c->d_m, c->d_v, c->d_in, c->d_h, c->d_o, c->d_col, c->d_gcol,
                   c->d_ga, c->d_gb, c->d_gh, c->d_go, c->d_part, c->d_res, c->d_tgt, c->d_loss, c->d_lossmean,
                   c->d_ones};
    for (float* p : fp) if (p) cudaFree(p);
    for (int l = 1; l <= NCONV; ++l) if (c->d_act[l]) cudaFree(c->d_act[l]);
    if (c->d_idx) cudaFree(c->d_idx);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

extern "C" long bsg_cnn_num_params(const bsg_cnn* h) {
    const Cnn* c = reinterpret_cast<const Cnn*>(h);
    return c ? c->nparams : 0;
}

extern "C" int bsg_cnn_get_params(bsg_cnn* h, float* out) {
    Cnn* c = reinterpret_cast<Cnn*>(h);
    if (!c || !out) return cfail(BSG_ERR_ARG, "bsg_cnn_get_params: null argument");
    CCK(cudaSetDevice(c->device));
    CCK(cudaMemcpy(out, c->d_w, sizeof(float) * c->nparams, cudaMemcpyDeviceToHost));
    return BSG_OK;
}

extern "C" int bsg_cnn_set_params(bsg_cnn* h, const float* in) {
    Cnn* c = reinterpret_cast<Cnn*>(h);
    if (!c || !in) return cfail(BSG_ERR_ARG, "bsg_cnn_set_params: null argument");
    CCK(cudaSetDevice(c->device));
    CCK(cudaMemcpy(c->d_w, in, sizeof(float) * c->nparams, cudaMemcpyHostToDevice));
    round_bf16_kernel<<<grid_for(c->nparams), 256, 0, c->stream>>>(c->d_w, c->d_weff, c->nparams);
    CCK(cudaGetLastError());
    CCK(cudaMemset(c->d_m, 0, sizeof(float) * c->nparams));
    CCK(cudaMemset(c->d_v, 0, sizeof(float) * c->nparams));
    c->step = 0;
    CCK(cudaStreamSynchronize(c->stream));
    return BSG_OK;
}

extern "C" int bsg_cnn_predict(bsg_cnn* h, const float* images, long n, float* out, int flags) {
    Cnn* c = reinterpret_cast<Cnn*>(h);
    if (!c || !images || !out || n < 1) return cfail(BSG_ERR_ARG, "bsg_cnn_predict: bad argument");
    CCK(cudaSetDevice(c->device));
    const int B = std::max(1, std::min<int>(c->cfg.batch > 0 ? c->cfg.batch : 256, (int)std::min<long>(n, 1 << 20)));
    int rc = ensure_batch(*c, B);
    if (rc) return rc;
    const int npix = c->cfg.box * c->cfg.box;
    cudaStream_t s = c->stream;
    float* d_src = nullptr;
    float* d_out = nullptr;
    if (!(flags & BSG_DEVICE_PTR)) {
        CCK(cudaMalloc(&d_src, sizeof(float) * (size_t)npix * B));
        CCK(cudaMalloc(&d_out, sizeof(float) * NRES * B));
    }
    cudaError_t e = cudaSuccess;
    for (long b0 = 0; e == cudaSuccess && b0 < n; b0 += B) {
        const int cnt = (int)std::min<long>(B, n - b0);
        const float* src = images + (size_t)b0 * npix;
        if (!(flags & BSG_DEVICE_PTR)) {
            e = cudaMemcpyAsync(d_src, src, sizeof(float) * (size_t)npix * cnt, cudaMemcpyHostToDevice, s);
            src = d_src;
        }
        if (e == cudaSuccess) { gather_norm_kernel<<<cnt, 256, 0, s>>>(src, nullptr, npix, c->d_in); e = cudaGetLastError(); }
        if (e == cudaSuccess) e = forward(*c, cnt, s);
        float* res = (flags & BSG_DEVICE_PTR) ? out + (size_t)b0 * NRES : d_out;
        if (e == cudaSuccess) {
            head_kernel<<<(cnt + 127) / 128, 128, 0, s>>>(c->d_o, cnt, nullptr, 0.f, res, nullptr, nullptr);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && !(flags & BSG_DEVICE_PTR))
            e = cudaMemcpyAsync(out + (size_t)b0 * NRES, d_out, sizeof(float) * NRES * cnt, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && !(flags & BSG_DEVICE_PTR)) e = cudaStreamSynchronize(s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_src);
    cudaFree(d_out);
    if (e != cudaSuccess) return cfail(BSG_ERR_CUDA, "bsg_cnn_predict: %s", cudaGetErrorString(e));
    return BSG_OK;
}

extern "C" int bsg_cnn_loss_grad(bsg_cnn* h, const float* images, const float* targets, long n, double* loss,
                                 float* grads) {
    Cnn* c = reinterpret_cast<Cnn*>(h);
    if (!c || !images || !targets || n < 1) return cfail(BSG_ERR_ARG, "bsg_cnn_loss_grad: bad argument");
    CCK(cudaSetDevice(c->device));
    const int B = (int)n;
    int rc = ensure_batch(*c, B);
    if (rc) return rc;
    const int npix = c->cfg.box * c->cfg.box;
    cudaStream_t s = c->stream;
    float* d_src = nullptr;
    CCK(cudaMalloc(&d_src, sizeof(float) * (size_t)npix * B));
    cudaError_t e = cudaMemcpyAsync(d_src, images, sizeof(float) * (size_t)npix * B, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->d_tgt, targets, sizeof(float) * NRES * B, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) { gather_norm_kernel<<<B, 256, 0, s>>>(d_src, nullptr, npix, c->d_in); e = cudaGetLastError(); }
    if (e == cudaSuccess) e = forward(*c, B, s);
    if (e == cudaSuccess) {
        head_kernel<<<(B + 127) / 128, 128, 0, s>>>(c->d_o, B, c->d_tgt, c->cfg.shift_weight, c->d_res, c->d_go, c->d_loss);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = backward(*c, B, s);
    std::vector<float> l(B);
    if (e == cudaSuccess) e = cudaMemcpyAsync(l.data(), c->d_loss, sizeof(float) * B, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && grads) e = cudaMemcpyAsync(grads, c->d_g, sizeof(float) * c->nparams, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_src);
    if (e != cudaSuccess) return cfail(BSG_ERR_CUDA, "bsg_cnn_loss_grad: %s", cudaGetErrorString(e));
    if (loss) {
        double t = 0;
        for (float v : l) t += v;
        *loss = t / B;
    }
    return BSG_OK;
}

extern "C" int bsg_cnn_train(bsg_cnn* h, const float* images, const float* targets, long ndata, int steps, float lr,
                             float* losses, int flags) {
    Cnn* c = reinterpret_cast<Cnn*>(h);
    if (!c || !images || !targets || ndata < 1 || steps < 1)
        return cfail(BSG_ERR_ARG, "bsg_cnn_train: bad argument");
    if (!(flags & BSG_DEVICE_PTR))
        return cfail(BSG_ERR_ARG, "bsg_cnn_train: the training set must be on the device (BSG_DEVICE_PTR)");
    CCK(cudaSetDevice(c->device));
    const int B = std::max(1, c->cfg.batch > 0 ? c->cfg.batch : 256);
    int rc = ensure_batch(*c, B);
    if (rc) return rc;
    const int npix = c->cfg.box * c->cfg.box;
    cudaStream_t s = c->stream;
    // mini-batch indices for every step (seeded, sampled without replacement
    // within each pass over the data)
    std::vector<int> idx((size_t)steps * B);
    std::mt19937_64 rng(c->cfg.seed + 7919ull * (uint64_t)c->step);
    std::vector<int> perm(ndata);
    long pos = ndata;
    for (size_t i = 0; i < idx.size(); ++i) {
        if (pos >= ndata) {
            for (long j = 0; j < ndata; ++j) perm[j] = (int)j;
            std::shuffle(perm.begin(), perm.end(), rng);
            pos = 0;
        }
        idx[i] = perm[pos++];
    }
    int* d_all = nullptr;
    float* d_losses = nullptr;
    CCK(cudaMalloc(&d_all, sizeof(int) * idx.size()));
    CCK(cudaMalloc(&d_losses, sizeof(float) * steps));
    cudaError_t e = cudaMemcpyAsync(d_all, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, s);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int t = 0; e == cudaSuccess && t < steps; ++t) {
        const int* bi = d_all + (size_t)t * B;
        gather_norm_kernel<<<B, 256, 0, s>>>(images, bi, npix, c->d_in);
        gather_rows_kernel<<<(B * NRES + 255) / 256, 256, 0, s>>>(targets, bi, B, NRES, c->d_tgt);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = forward(*c, B, s);
        if (e == cudaSuccess) {
            head_kernel<<<(B + 127) / 128, 128, 0, s>>>(c->d_o, B, c->d_tgt, c->cfg.shift_weight, c->d_res, c->d_go,
                                                        c->d_loss);
            mean_kernel<<<1, 32, 0, s>>>(c->d_loss, B, d_losses + t);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = backward(*c, B, s);
        if (e == cudaSuccess) {
            ++c->step;
            const float c1 = 1.f / (1.f - powf(b1, (float)c->step)), c2 = 1.f / (1.f - powf(b2, (float)c->step));
            adam_kernel<<<grid_for(c->nparams), 256, 0, s>>>(c->d_w, c->d_weff, c->d_g, c->d_m, c->d_v, c->nparams, lr,
                                                             b1, b2, eps, c1, c2);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess && losses) e = cudaMemcpyAsync(losses, d_losses, sizeof(float) * steps, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_all);
    cudaFree(d_losses);
    if (e != cudaSuccess) return cfail(BSG_ERR_CUDA, "bsg_cnn_train: %s", cudaGetErrorString(e));
    return BSG_OK;
}

namespace bsg {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// per image: variance of the signal inside the inscribed circle, then
// Gaussian noise of variance var / snr (Box-Muller on a counter-based hash
// of seed, image and pixel, so the result does not depend on the launch)
__global__ void __launch_bounds__(256) add_noise_kernel(float* __restrict__ img, int box, double snr, uint64_t seed) {
    __shared__ double s1[256], s2[256], s3[256];
    float* p = img + (size_t)blockIdx.x * box * box;
    const double c = box / 2.0, r2 = c * c;
    double a = 0, b = 0, n = 0;
    for (int i = threadIdx.x; i < box * box; i += 256) {
        const double dx = i % box - c, dy = i / box - c;
        if (dx * dx + dy * dy <= r2) { const double v = p[i]; a += v; b += v * v; n += 1; }
    }
    s1[threadIdx.x] = a; s2[threadIdx.x] = b; s3[threadIdx.x] = n;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if (threadIdx.x < o) {
            s1[threadIdx.x] += s1[threadIdx.x + o]; s2[threadIdx.x] += s2[threadIdx.x + o]; s3[threadIdx.x] += s3[threadIdx.x + o];
        }
        __syncthreads();
    }
    const double mean = s1[0] / s3[0], var = s2[0] / s3[0] - mean * mean;
    const double sd = var > 0 ? sqrt(var / snr) : 0.0;
    for (int i = threadIdx.x; i < box * box; i += 256) {
        const uint64_t h = mix64(seed ^ mix64(((uint64_t)blockIdx.x << 32) + (uint64_t)i + 0x9E3779B97F4A7C15ull));
        const double u1 = ((h >> 11) + 1.0) / 9007199254740993.0;
        const double u2 = (mix64(h) >> 11) / 9007199254740992.0;
        p[i] += (float)(sd * sqrt(-2.0 * log(u1)) * cos(2 * M_PI * u2));
    }
}

}  // namespace
}  // namespace bsg

extern "C" int bsg_add_noise(float* d_images, long n, int box, double snr, unsigned long long seed, void* stream) {
    if (!d_images || n < 1 || box < 2 || !(snr > 0)) return cfail(BSG_ERR_ARG, "bsg_add_noise: bad argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (long b0 = 0; b0 < n; b0 += 65535) {
        const long cnt = std::min(65535L, n - b0);
        add_noise_kernel<<<(unsigned)cnt, 256, 0, s>>>(d_images + (size_t)b0 * box * box, box, snr, seed + (uint64_t)b0);
        CCK(cudaGetLastError());
    }
    CCK(cudaStreamSynchronize(s));
    return BSG_OK;
}
