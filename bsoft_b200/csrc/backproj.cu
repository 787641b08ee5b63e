// backproj.cu - real-space weighted back-projection (bbackproj:
// project_back_projection, bsoft/src/mg/mg_reconstruct.cpp:1524-1624, over
// Bimage::back_project, bsoft/src/img/Bimage_project.cpp:466-509).
//
// Per image, as the reference does it:
//   * fspace_weigh_ramp (bsoft/src/img/Bimage_fspace.cpp:1220-1268): forward
//     2-D transform, every coefficient times |s| (s = k / real size per axis,
//     k folded at the integer half size) or 0 beyond the resolution limit,
//     inverse transform, real part.  Three passes here: the rows forward, the
//     columns (forward, ramp, inverse, in shared memory), the rows inverse with
//     the real part and per-row FP64 moments;
//   * rescale_to_avg_std(0, 1) from the filtered image's average and
//     population standard deviation, stored as float, and the background (the
//     mean outside the ellipse about the image origin, calculate_background,
//     Bimage_background.cpp:27-80) as the fill: one CTA per image;
//   * every map voxel c (relative to the map's origin, its integer half size)
//     adds the image sampled at diag(mag, mag, 1) M^T c + origin (z dropped)
//     with Bimage::interpolate (bsoft/src/img/Bimage.cpp:1436-1484: bilinear in
//     the image plane with its weight flips, the sum divided by the sum of the
//     weights, the fill outside), the map stored as float after every image,
//     in image order.
//
// The map accumulators are float, as the reference's map is; images go to
// one of two maps when half maps are asked for.  The back-projection kernel
// runs one thread per voxel over a batch of images whose parameters sit in
// shared memory and whose pixels are read through the read-only cache (a
// batch's images fit in L2); coordinates, weights and the division are FP64
// with explicit round-to-nearest operations in the reference's order.
#include "context.cuh"
#include "fft_dev.cuh"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <vector>

namespace bsg {

cudaError_t launch_symmetrize(const Context& c, float* map, float* tmp, bool sinc, cudaStream_t s);
cudaError_t launch_rescale(const Context& c, float* map, double nuavg, double nustd, bool sinc, cudaStream_t s);

namespace {

struct BpImage {
    double m[6];        // rows 0 and 1 of diag(mag, mag, 1) M^T: image x, y of a map offset
    double ox, oy;      // image origin (pixels)
    double fill;        // background of the rescaled image (written by norm_kernel)
    double inv_real;    // 1 / (n * pixel): frequency per index of the ramp
    double s2max;       // 1 / resolution^2 after the image's check_resolution
    int map;            // half-map index 0 / 1
    int pad;
};

struct FftPlan {
    int mixed;          // 0: power of two (radix-2/4 on bit-reversed input); 1: Stockham
    int log;            // log2(n) for the power-of-two path
    int nstage;
    int r[16];
};

constexpr int XW = 8;               // row lines (warps) per CTA

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// One warp transforms the line in buf (n values; 2n of room for the mixed
// path), input order as the path wants it.
template <bool INV>
__device__ __forceinline__ void line_fft(float2* buf, int n, const FftPlan& p, const float2* roots) {
    if (p.mixed) warp_fft_mixed<INV>(buf, buf + n, n, p.r, p.nstage, roots);
    else warp_fft<INV>(buf, n, p.log, roots);
}

// Rows forward: real image rows -> complex spectra rows (work).
__global__ void __launch_bounds__(XW * 32) rows_fwd_kernel(const float* img, float2* work, int n, long lines,
                                                            const float2* roots, FftPlan p) {
    extern __shared__ float2 sm[];
    float2* sroot = sm;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = p.mixed ? 2 * n : n;
    float2* buf = sm + n + warp * per;
    for (int i = threadIdx.x; i < n; i += blockDim.x) sroot[i] = roots[i];
    __syncthreads();
    const long line = (long)blockIdx.x * XW + warp;
    if (line >= lines) return;
    const float* src = img + line * n;
    for (int i = lane; i < n; i += 32) {
        const int at = p.mixed ? i : (int)bitrev((unsigned)i, p.log);
        buf[at] = make_float2(src[i], 0.f);
    }
    __syncwarp();
    line_fft<false>(buf, n, p, sroot);
    float2* dst = work + line * n;
    for (int i = lane; i < n; i += 32) dst[i] = buf[i];
}

// Columns: forward transform along y, the ramp |s| (0 beyond s2max) times
// 1/n^2 (both of the reference's 1/sqrt(n^2) normalisations), inverse along y.
// CTA: `cw` adjacent columns of one image (blockIdx.y).
__global__ void cols_kernel(float2* work, const BpImage* par, int n, int cw, double norm, const float2* roots,
                            FftPlan p) {
    extern __shared__ float2 sm[];
    float2* sroot = sm;
    const int per = p.mixed ? 2 * n : n;
    float2* tile = sm + n;               // cw lines of `per`
    for (int i = threadIdx.x; i < n; i += blockDim.x) sroot[i] = roots[i];
    const int x0 = blockIdx.x * cw;
    float2* base = work + (size_t)blockIdx.y * n * n;
    for (int i = threadIdx.x; i < cw * n; i += blockDim.x) {
        const int c = i % cw, j = i / cw;
        const int x = x0 + c;
        float2 v = make_float2(0.f, 0.f);
        if (x < n) v = base[(size_t)j * n + x];
        tile[c * per + (p.mixed ? j : (int)bitrev((unsigned)j, p.log))] = v;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int x = x0 + warp;
    if (warp < cw && x < n) {
        float2* buf = tile + warp * per;
        line_fft<false>(buf, n, p, sroot);
        // fspace_weigh_ramp: k folded at h = n / 2 on both axes
        const double inv_real = par[blockIdx.y].inv_real, s2max = par[blockIdx.y].s2max;
        const int h = n / 2;
        const double sx = (double)(x > h ? n - x : x) * inv_real;
        for (int j = lane; j < n; j += 32) {
            const double sy = (double)(j > h ? n - j : j) * inv_real;
            const double s2 = sx * sx + sy * sy;
            const double w = s2 > s2max ? 0.0 : sqrt(s2) * norm;
            const float2 v = buf[j];
            buf[j] = make_float2((float)(v.x * w), (float)(v.y * w));
        }
        __syncwarp();
        if (!p.mixed) {
            // the power-of-two path wants bit-reversed input again
            for (int j = lane; j < n; j += 32) {
                const int r = (int)bitrev((unsigned)j, p.log);
                if (j < r) { const float2 a = buf[j]; buf[j] = buf[r]; buf[r] = a; }
            }
            __syncwarp();
        }
        line_fft<true>(buf, n, p, sroot);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < cw * n; i += blockDim.x) {
        const int c = i % cw, j = i / cw;
        const int xx = x0 + c;
        if (xx < n) base[(size_t)j * n + xx] = tile[c * per + j];
    }
}

// Rows inverse: complex rows -> real part (float image) and the row's FP64
// sums of v and v^2 (Bimage::statistics over the float values).
__global__ void __launch_bounds__(XW * 32) rows_inv_kernel(const float2* work, float* img, double* rowsum, int n,
                                                            long lines, const float2* roots, FftPlan p) {
    extern __shared__ float2 sm[];
    float2* sroot = sm;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = p.mixed ? 2 * n : n;
    float2* buf = sm + n + warp * per;
    for (int i = threadIdx.x; i < n; i += blockDim.x) sroot[i] = roots[i];
    __syncthreads();
    const long line = (long)blockIdx.x * XW + warp;
    if (line >= lines) return;
    const float2* src = work + line * n;
    for (int i = lane; i < n; i += 32) buf[p.mixed ? i : (int)bitrev((unsigned)i, p.log)] = src[i];
    __syncwarp();
    line_fft<true>(buf, n, p, sroot);
    float* dst = img + line * n;
    double s1 = 0, s2 = 0;
    for (int i = lane; i < n; i += 32) {
        const float v = buf[i].x;
        dst[i] = v;
        s1 += (double)v;
        s2 += (double)v * (double)v;
    }
    for (int o = 16; o; o >>= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
        rowsum[2 * line] = s1;
        rowsum[2 * line + 1] = s2;
    }
}

// One CTA per image: average and standard deviation from the row sums,
// v -> float(v scale + shift) with scale = 1/std (1 if std <= 1e-30), shift =
// -avg scale (Bimage::rescale_to_avg_std, Bimage_rescale.cpp:163-182), and the
// fill: the mean of the rescaled pixels with ((x-ox)/hx)^2 + ((y-oy)/hy)^2 > 1,
// hx = hy = n / 2 (calculate_background of a 2-D image).
__global__ void norm_kernel(float* img, const double* rowsum, BpImage* par, int n) {
    __shared__ double ra[256], rb[256];
    __shared__ long rc[256];
    __shared__ double sc[2];
    const int k = blockIdx.x;
    float* p = img + (size_t)k * n * n;
    double a = 0, b = 0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        a += rowsum[2 * ((size_t)k * n + r)];
        b += rowsum[2 * ((size_t)k * n + r) + 1];
    }
    ra[threadIdx.x] = a;
    rb[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s; s >>= 1) {
        if ((int)threadIdx.x < s) {
            ra[threadIdx.x] += ra[threadIdx.x + s];
            rb[threadIdx.x] += rb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double np = (double)n * n;
        const double avg = ra[0] / np;
        double var = rb[0] / np - avg * avg;
        const double sd = var > 0 ? sqrt(var) : 0.0;
        const double scale = sd > 1e-30 ? 1.0 / sd : 1.0;
        sc[0] = scale;
        sc[1] = 0.0 - avg * scale;
    }
    __syncthreads();
    const double scale = sc[0], shift = sc[1];
    const double ox = par[k].ox, oy = par[k].oy, hh = (double)(n / 2);
    double bs = 0;
    long bc = 0;
    for (long i = threadIdx.x; i < (long)n * n; i += blockDim.x) {
        const float v = (float)dadd(dmul((double)p[i], scale), shift);
        p[i] = v;
        const long x = i % n, y = i / n;
        double x2 = __ddiv_rn(dsub((double)x, ox), hh), y2 = __ddiv_rn(dsub((double)y, oy), hh);
        x2 = dmul(x2, x2);
        y2 = dmul(y2, y2);
        if (dsub(dadd(x2, y2), 1.0) > 0) {
            bs += (double)v;
            ++bc;
        }
    }
    __syncthreads();
    ra[threadIdx.x] = bs;
    rc[threadIdx.x] = bc;
    __syncthreads();
    for (int s = blockDim.x / 2; s; s >>= 1) {
        if ((int)threadIdx.x < s) {
            ra[threadIdx.x] += ra[threadIdx.x + s];
            rc[threadIdx.x] += rc[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) par[k].fill = rc[0] ? ra[0] / (double)rc[0] : 0.0;
}

// Bimage::interpolate of a one-plane image at (x, y, 0): the z loop keeps only
// the plane with weight 1; the y and x weights flip once per visited sample,
// the x flips not reset between rows.
__device__ __forceinline__ double interpolate2(const float* __restrict__ im, int n, double x, double y,
                                               double fill) {
    if (!(x >= 0 && x < n && y >= 0 && y < n)) return fill;
    const int ix = (int)x, iy = (int)y;
    const int cx = n < ix + 2 ? 1 : 2, cy = n < iy + 2 ? 1 : 2;
    double fx = dsub(x, (double)ix), fy = dsub(y, (double)iy);
    double value = 0, ws = 0;
#pragma unroll
    for (int yk = 0; yk < 2; ++yk) {
        const bool ay = yk < cy;
        if (ay) fy = dsub(1.0, fy);
        const double wy = fy;            // fy * fz with fz = 1 - 0 = 1
#pragma unroll
        for (int xk = 0; xk < 2; ++xk) {
            const bool ax = ay && xk < cx;
            if (ax) {
                fx = dsub(1.0, fx);
                const double w = dmul(fx, wy);
                const int yy = min(iy + yk, n - 1), xx = min(ix + xk, n - 1);
                ws = dadd(ws, w);
                value = dadd(value, dmul((double)__ldg(im + (size_t)yy * n + xx), w));
            }
        }
    }
    return ws != 0 ? __ddiv_rn(value, ws) : fill;
}

constexpr int BP_THREADS = 128;
constexpr int BP_CHUNK = 64;         // image parameters staged in shared memory at a time

// One thread per voxel (x fastest), every image of the batch in order; the
// map(s) read once and written once per batch.
__global__ void __launch_bounds__(BP_THREADS) backproject_kernel(const float* __restrict__ img,
                                                                 const BpImage* __restrict__ par, int nimg, int n,
                                                                 int N, float* map0, float* map1) {
    __shared__ BpImage sp[BP_CHUNK];
    const int x = blockIdx.x * BP_THREADS + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    const bool live = x < N;
    const size_t i = ((size_t)z * N + y) * N + (live ? x : 0);
    const double o = (double)(N / 2);
    const double c0 = dsub((double)x, o), c1 = dsub((double)y, o), c2 = dsub((double)z, o);
    float acc0 = live ? map0[i] : 0.f;
    float acc1 = (live && map1) ? map1[i] : 0.f;
    const size_t n2 = (size_t)n * n;
    for (int k0 = 0; k0 < nimg; k0 += BP_CHUNK) {
        const int cnt = min(BP_CHUNK, nimg - k0);
        __syncthreads();
        for (int t = threadIdx.x; t < cnt; t += blockDim.x) sp[t] = par[k0 + t];
        __syncthreads();
        if (!live) continue;
        for (int t = 0; t < cnt; ++t) {
            const BpImage& q = sp[t];
            // mat * newcoor + oldorigin, row by row
            const double X = dadd(dadd(dadd(dmul(q.m[0], c0), dmul(q.m[1], c1)), dmul(q.m[2], c2)), q.ox);
            const double Y = dadd(dadd(dadd(dmul(q.m[3], c0), dmul(q.m[4], c1)), dmul(q.m[5], c2)), q.oy);
            const double v = interpolate2(img + (size_t)(k0 + t) * n2, n, X, Y, q.fill);
            if (q.map) acc1 = (float)dadd((double)acc1, v);
            else acc0 = (float)dadd((double)acc0, v);
        }
    }
    if (live) {
        map0[i] = acc0;
        if (map1) map1[i] = acc1;
    }
}

// dst = a + b, float additions
__global__ void add_maps_kernel(float* dst, const float* a, const float* b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = __fadd_rn(a[i], b[i]);
}

thread_local char g_bp_err[512] = "";

int bp_fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_bp_err, sizeof(g_bp_err), fmt, ap);
    va_end(ap);
    set_error("%s", g_bp_err);
    return code;
}

FftPlan fft_plan_for(int n) {
    FftPlan p{};
    p.mixed = (n & (n - 1)) != 0;
    if (p.mixed) p.nstage = factor_radices(n, p.r);
    else p.log = ilog2i(n);
    return p;
}

}  // namespace
}  // namespace bsg

struct bsg_backproj {
    bsg_backproj_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    int halves = 0;                   // 1: two accumulators (half maps)
    bsg::FftPlan fp{};
    int cw = 16;                      // columns per CTA of cols_kernel
    float* d_map[2] = {nullptr, nullptr};
    float* d_out = nullptr;           // finished map
    float* d_tmp = nullptr;           // symmetrization work map
    float* d_img = nullptr;           // batch x n^2
    float2* d_work = nullptr;         // batch x n^2
    double* d_rowsum = nullptr;       // batch x n x 2
    bsg::BpImage* d_par = nullptr;
    float2* d_roots = nullptr;        // n roots exp(-2 pi i t / n)
    std::vector<bsg::BpImage> h_par;
    bsg::Context ctx;                 // map geometry and -symmetry for the shared finishing kernels
    double rescale_avg = 0, rescale_std = 0;
    long images = 0;
};

namespace {

void bp_free(bsg_backproj* b) {
    auto F = [](void* p) { if (p) cudaFree(p); };
    F(b->d_map[0]); F(b->d_map[1]); F(b->d_out); F(b->d_tmp); F(b->d_img); F(b->d_work); F(b->d_rowsum);
    F(b->d_par); F(b->d_roots);
    if (b->stream) cudaStreamDestroy(b->stream);
}

#define BP_CK(call)                                                                                      \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return bsg::bp_fail(BSG_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                                __LINE__);                                                               \
    } while (0)

size_t row_smem(int n, const bsg::FftPlan& p) {
    return sizeof(float2) * ((size_t)n + (size_t)bsg::XW * (p.mixed ? 2 * n : n));
}

size_t col_smem(int n, int cw, const bsg::FftPlan& p) {
    return sizeof(float2) * ((size_t)n + (size_t)cw * (p.mixed ? 2 * n : n));
}

}  // namespace

extern "C" {

int bsg_backproj_create(const bsg_backproj_config* cfg, bsg_backproj** out) {
    using namespace bsg;
    if (!cfg || !out) return bp_fail(BSG_ERR_ARG, "bsg_backproj_create: null argument");
    *out = nullptr;
    const int n = cfg->n, N = cfg->map;
    if (n < 2 || n > 1024) return bp_fail(BSG_ERR_ARG, "bsg_backproj_create: image edge %d outside 2..1024", n);
    FftPlan fp = fft_plan_for(n);
    if (fp.mixed && fp.nstage < 0)
        return bp_fail(BSG_ERR_ARG, "bsg_backproj_create: image edge %d has a prime factor above 7", n);
    if (N < 2 || N > 1024) return bp_fail(BSG_ERR_ARG, "bsg_backproj_create: map edge %d outside 2..1024", N);
    if (!(cfg->pixel > 0)) return bp_fail(BSG_ERR_ARG, "bsg_backproj_create: pixel size must be positive");
    if (cfg->nmaps < 1 || cfg->nmaps > 3) return bp_fail(BSG_ERR_ARG, "bsg_backproj_create: nmaps must be 1, 2 or 3");
    int dev = cfg->device, ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return bp_fail(BSG_ERR_NODEV, "bsg_backproj_create: no CUDA device");
    if (dev < 0 || dev >= ndev) return bp_fail(BSG_ERR_ARG, "bsg_backproj_create: device %d of %d", dev, ndev);
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess || prop.major != 10)
        return bp_fail(BSG_ERR_NODEV, "bsg_backproj_create: device %d is not sm_100", dev);
    bsg_backproj* b = new (std::nothrow) bsg_backproj();
    if (!b) return bp_fail(BSG_ERR_NOMEM, "bsg_backproj_create: host allocation");
    b->cfg = *cfg;
    b->device = dev;
    b->fp = fp;
    b->halves = (cfg->nmaps & 2) ? 1 : 0;
    if (b->cfg.batch <= 0) b->cfg.batch = 256;
    b->cfg.batch = std::min(b->cfg.batch, 4096);
    // columns per CTA: 16 while the tile fits in shared memory
    b->cw = 16;
    while (b->cw > 1 && col_smem(n, b->cw, fp) > 200 * 1024) b->cw /= 2;
    b->ctx.g.map = N;
    int rc = BSG_OK;
    auto A = [&](void** p, size_t bytes) {
        if (rc) return;
        if (cudaMalloc(p, bytes) != cudaSuccess) rc = bp_fail(BSG_ERR_NOMEM, "bsg_backproj_create: %zu bytes", bytes);
    };
    if (cudaSetDevice(dev) != cudaSuccess) { delete b; return bp_fail(BSG_ERR_CUDA, "bsg_backproj_create: set device"); }
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return bp_fail(BSG_ERR_CUDA, "bsg_backproj_create: stream");
    }
    const size_t N3 = (size_t)N * N * N, B = (size_t)b->cfg.batch, n2 = (size_t)n * n;
    A((void**)&b->d_map[0], sizeof(float) * N3);
    if (b->halves) A((void**)&b->d_map[1], sizeof(float) * N3);
    A((void**)&b->d_out, sizeof(float) * N3);
    A((void**)&b->d_img, sizeof(float) * B * n2);
    A((void**)&b->d_work, sizeof(float2) * B * n2);
    A((void**)&b->d_rowsum, sizeof(double) * 2 * B * n);
    A((void**)&b->d_par, sizeof(BpImage) * B);
    A((void**)&b->d_roots, sizeof(float2) * n);
    if (rc) { bp_free(b); delete b; return rc; }
    std::vector<float2> roots(n);
    for (int t = 0; t < n; ++t) {
        const double a = -2.0 * M_PI * t / n;
        roots[t] = make_float2((float)cos(a), (float)sin(a));
    }
    cudaError_t e = cudaMemcpy(b->d_roots, roots.data(), sizeof(float2) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_map[0], 0, sizeof(float) * N3, b->stream);
    if (e == cudaSuccess && b->halves) e = cudaMemsetAsync(b->d_map[1], 0, sizeof(float) * N3, b->stream);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(cols_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem(n, b->cw, fp));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(rows_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)row_smem(n, fp));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(rows_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)row_smem(n, fp));
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) {
        bp_free(b);
        delete b;
        return bp_fail(BSG_ERR_CUDA, "bsg_backproj_create: %s", cudaGetErrorString(e));
    }
    *out = b;
    return BSG_OK;
}

void bsg_backproj_destroy(bsg_backproj* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    bp_free(b);
    delete b;
}

int bsg_backproj_add(bsg_backproj* b, const float* images, const double* records, long count, int flags) {
    using namespace bsg;
    if (!b) return bp_fail(BSG_ERR_ARG, "bsg_backproj_add: null context");
    if (count < 0 || (count > 0 && (!images || !records))) return bp_fail(BSG_ERR_ARG, "bsg_backproj_add: bad arguments");
    const int n = b->cfg.n, N = b->cfg.map;
    const size_t n2 = (size_t)n * n;
    const bool on_dev = (flags & BSG_DEVICE_PTR) != 0;
    if (on_dev) {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, images) != cudaSuccess || at.type != cudaMemoryTypeDevice)
            return bp_fail(BSG_ERR_ARG, "bsg_backproj_add: BSG_DEVICE_PTR given but images are not device memory");
    }
    BP_CK(cudaSetDevice(b->device));
    for (long k = 0; k < count; ++k) {
        const double* q = records + k * BSG_BACKPROJ_DOUBLES;
        const int m = (int)q[12];
        if (!(q[11] > 0)) return bp_fail(BSG_ERR_ARG, "bsg_backproj_add: record %ld: magnification must be positive", k);
        if (m < 0 || m > 1 || (m == 1 && !b->halves))
            return bp_fail(BSG_ERR_ARG, "bsg_backproj_add: record %ld: map index %d with %s", k, m,
                           b->halves ? "half maps" : "one map");
        if (q[13] < 0) return bp_fail(BSG_ERR_ARG, "bsg_backproj_add: record %ld: negative pixel size", k);
        for (int j = 0; j < 14; ++j)
            if (!isfinite(q[j])) return bp_fail(BSG_ERR_ARG, "bsg_backproj_add: record %ld field %d not finite", k, j);
    }
    const long B = b->cfg.batch;
    b->h_par.resize((size_t)B);
    for (long k0 = 0; k0 < count; k0 += B) {
        const long cnt = std::min(B, count - k0);
        for (long k = 0; k < cnt; ++k) {
            const double* q = records + (k0 + k) * BSG_BACKPROJ_DOUBLES;
            BpImage& p = b->h_par[(size_t)k];
            memset(&p, 0, sizeof(p));
            // mat = diag(mag, mag, 1) * M^T (Bimage_project.cpp:486-488): row r of
            // M^T is column r of M, rows 0 and 1 scaled by the magnification
            const double* M = q + 2;
            const double mag = q[11];
            for (int r = 0; r < 2; ++r)
                for (int c = 0; c < 3; ++c) p.m[3 * r + c] = M[3 * c + r] * mag;
            p.ox = q[0];
            p.oy = q[1];
            p.map = (int)q[12];
            // Bimage::check_resolution of the image (two axes of pixel u): at
            // most its real size, at least 2 / sqrt(2 / u^2)
            const double u = q[13] > 0 ? q[13] : b->cfg.pixel, real = n * u;
            double res = b->cfg.resolution;
            if (res > real) res = real;
            else res = std::max(res, 2.0 / sqrt(1.0 / (u * u) + 1.0 / (u * u)));
            p.inv_real = 1.0 / real;
            p.s2max = 1.0 / (res * res);
        }
        const float* src = images + (size_t)k0 * n2;
        BP_CK(cudaMemcpyAsync(b->d_img, src, sizeof(float) * n2 * cnt,
                              on_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, b->stream));
        BP_CK(cudaMemcpyAsync(b->d_par, b->h_par.data(), sizeof(BpImage) * cnt, cudaMemcpyHostToDevice, b->stream));
        const long lines = cnt * n;
        const unsigned rblocks = (unsigned)((lines + XW - 1) / XW);
        rows_fwd_kernel<<<rblocks, XW * 32, row_smem(n, b->fp), b->stream>>>(b->d_img, b->d_work, n, lines,
                                                                             b->d_roots, b->fp);
        BP_CK(cudaGetLastError());
        const dim3 cg((unsigned)((n + b->cw - 1) / b->cw), (unsigned)cnt);
        cols_kernel<<<cg, b->cw * 32, col_smem(n, b->cw, b->fp), b->stream>>>(
            b->d_work, b->d_par, n, b->cw, 1.0 / ((double)n * n), b->d_roots, b->fp);
        BP_CK(cudaGetLastError());
        rows_inv_kernel<<<rblocks, XW * 32, row_smem(n, b->fp), b->stream>>>(b->d_work, b->d_img, b->d_rowsum, n,
                                                                             lines, b->d_roots, b->fp);
        BP_CK(cudaGetLastError());
        norm_kernel<<<(unsigned)cnt, 256, 0, b->stream>>>(b->d_img, b->d_rowsum, b->d_par, n);
        BP_CK(cudaGetLastError());
        const dim3 g((unsigned)((N + BP_THREADS - 1) / BP_THREADS), (unsigned)N, (unsigned)N);
        backproject_kernel<<<g, BP_THREADS, 0, b->stream>>>(b->d_img, b->d_par, (int)cnt, n, N, b->d_map[0],
                                                           b->halves ? b->d_map[1] : nullptr);
        BP_CK(cudaGetLastError());
        // the staging buffers are reused by the next batch; host inputs must
        // stay valid until the copies are done
        BP_CK(cudaStreamSynchronize(b->stream));
        b->images += cnt;
    }
    return BSG_OK;
}

int bsg_backproj_set_symmetrize(bsg_backproj* b, const double* axes, const int* orders, int nops) {
    if (!b) return bsg::bp_fail(BSG_ERR_ARG, "bsg_backproj_set_symmetrize: null context");
    if (nops < 0 || (nops > 0 && (!axes || !orders)))
        return bsg::bp_fail(BSG_ERR_ARG, "bsg_backproj_set_symmetrize: bad arguments");
    for (int i = 0; i < nops; ++i)
        if (orders[i] < 1 || orders[i] > 9)
            return bsg::bp_fail(BSG_ERR_ARG, "bsg_backproj_set_symmetrize: order %d outside 1..9", orders[i]);
    b->ctx.symz_axes.assign(axes, axes + 3 * nops);
    b->ctx.symz_orders.assign(orders, orders + nops);
    return BSG_OK;
}

int bsg_backproj_set_rescale(bsg_backproj* b, double avg, double std) {
    if (!b) return bsg::bp_fail(BSG_ERR_ARG, "bsg_backproj_set_rescale: null context");
    b->rescale_avg = avg;
    b->rescale_std = std > 0 ? std : 0;
    return BSG_OK;
}

int bsg_backproj_finish(bsg_backproj* b, int imap, float* map_out, int flags) {
    using namespace bsg;
    if (!b || !map_out) return bp_fail(BSG_ERR_ARG, "bsg_backproj_finish: null argument");
    if (imap < 0 || imap > 2 || (imap > 0 && !b->halves))
        return bp_fail(BSG_ERR_ARG, "bsg_backproj_finish: map %d not available with nmaps %d", imap, b->cfg.nmaps);
    const int N = b->cfg.map;
    const size_t N3 = (size_t)N * N * N;
    BP_CK(cudaSetDevice(b->device));
    // img_backprojection_accumulate (mg_reconstruct.cpp:1640-1684): the full
    // map is the float sum of the partial maps, a half map its own
    if (imap == 0 && b->halves) {
        add_maps_kernel<<<148 * 8, 256, 0, b->stream>>>(b->d_out, b->d_map[0], b->d_map[1], N3);
        BP_CK(cudaGetLastError());
    } else {
        const float* src = b->d_map[imap == 2 ? 1 : 0];
        BP_CK(cudaMemcpyAsync(b->d_out, src, sizeof(float) * N3, cudaMemcpyDeviceToDevice, b->stream));
    }
    if (!b->ctx.symz_orders.empty()) {
        if (!b->d_tmp && cudaMalloc((void**)&b->d_tmp, sizeof(float) * N3) != cudaSuccess)
            return bp_fail(BSG_ERR_NOMEM, "bsg_backproj_finish: work map");
        BP_CK(launch_symmetrize(b->ctx, b->d_out, b->d_tmp, false, b->stream));
    }
    if (b->rescale_std > 0) BP_CK(launch_rescale(b->ctx, b->d_out, b->rescale_avg, b->rescale_std, false, b->stream));
    BP_CK(cudaMemcpyAsync(map_out, b->d_out, sizeof(float) * N3,
                          (flags & BSG_DEVICE_PTR) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, b->stream));
    BP_CK(cudaStreamSynchronize(b->stream));
    return BSG_OK;
}

int bsg_backproj_reset(bsg_backproj* b) {
    if (!b) return bsg::bp_fail(BSG_ERR_ARG, "bsg_backproj_reset: null context");
    const size_t N3 = (size_t)b->cfg.map * b->cfg.map * b->cfg.map;
    BP_CK(cudaSetDevice(b->device));
    BP_CK(cudaMemsetAsync(b->d_map[0], 0, sizeof(float) * N3, b->stream));
    if (b->halves) BP_CK(cudaMemsetAsync(b->d_map[1], 0, sizeof(float) * N3, b->stream));
    BP_CK(cudaStreamSynchronize(b->stream));
    b->images = 0;
    return BSG_OK;
}

}  // extern "C"
