// symmetrize.cu - point-group symmetrization of a finished map in real
// space (breconstruct -mode 1: Bimage::symmetrize(sym, 1) after fft_back,
// bsoft/src/breconstruct.cpp:335, bsoft/src/img/Bimage_symmetry.cpp:31-100).
//
// For each generating operation (axis, order k) of the group, in Bsymmetry's
// order, the map becomes the float sum of itself and its k - 1 rotations by
// j 2 pi / k about the axis through the map origin (N/2, N/2, N/2); a
// rotation resamples the map with Bimage::interpolate
// (bsoft/src/img/Bimage.cpp:1436-1484): trilinear over the neighbours inside
// the map, its fractional weights flipped once per visited sample and not
// reset between rows (so at the upper edge, where a sample has one
// neighbour along an axis, the later rows take the unflipped weight), the
// sum divided by the sum of the weights, the map's background (the mean
// outside the inscribed ellipsoid, Bimage::calculate_background,
// bsoft/src/img/Bimage_background.cpp:27-80) where the sample falls outside
// or no weight remains, and the result stored as float.  At the end every
// value is multiplied by 1 / (group order).
//
// Every floating-point step uses an explicit round-to-nearest intrinsic, in
// the reference's order, so no multiply-add is contracted: the result is the
// reference's to the bit wherever the background sum (a fixed-order FP64
// reduction here, a running sum there) does not enter.
#include "context.cuh"

#include <math.h>

#include <vector>

namespace bsg {

namespace {

constexpr int MAXROT = 8;          // rotations per operation (orders up to 9)

struct RotArgs {
    const float* src;
    float* dst;
    int N;
    int nrot;                      // k - 1
    double m[MAXROT][9];           // row-major rotation matrices
    double o;                      // origin (N / 2) on every axis
    double fill;
};

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// Bimage::interpolate of src at (x, y, z)
__device__ double interpolate(const float* src, int N, double x, double y, double z, double fill) {
    if (!(x >= 0 && x < N && y >= 0 && y < N && z >= 0 && z < N)) return fill;
    const long ix = (long)x, iy = (long)y, iz = (long)z;
    const int cx = N < ix + 2 ? 1 : 2, cy = N < iy + 2 ? 1 : 2, cz = N < iz + 2 ? 1 : 2;
    double fx = dsub(x, (double)ix), fy = dsub(y, (double)iy), fz = dsub(z, (double)iz);
    double value = 0, ws = 0;
    for (int zk = 0; zk < 2; ++zk) {
        const bool az = zk < cz;
        if (az) fz = dsub(1.0, fz);
        for (int yk = 0; yk < 2; ++yk) {
            const bool ay = az && yk < cy;
            if (ay) fy = dsub(1.0, fy);
            const double wyz = dmul(fy, fz);
            for (int xk = 0; xk < 2; ++xk) {
                const bool ax = ay && xk < cx;
                if (ax) fx = dsub(1.0, fx);
                if (ax) {
                    const double w = dmul(fx, wyz);
                    const long zz = min(iz + zk, (long)N - 1), yy = min(iy + yk, (long)N - 1),
                               xx = min(ix + xk, (long)N - 1);
                    ws = dadd(ws, w);
                    value = dadd(value, dmul((double)src[(zz * N + yy) * N + xx], w));
                }
            }
        }
    }
    return ws != 0 ? __ddiv_rn(value, ws) : fill;
}

// dst = src + sum_j rotation_j(src), float additions in order j = 1 .. k-1
__global__ void rotate_sum_kernel(RotArgs a) {
    const long N = a.N, N3 = N * N * N;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N3; i += (long)gridDim.x * blockDim.x) {
        const long xx = i % N, yy = (i / N) % N, zz = i / (N * N);
        const double n0 = dsub((double)xx, a.o), n1 = dsub((double)yy, a.o), n2 = dsub((double)zz, a.o);
        float acc = a.src[i];
        for (int r = 0; r < a.nrot; ++r) {
            const double* M = a.m[r];
            // old = M^T nu + origin, as ((n0 M0i + n1 M1i) + n2 M2i) + o
            const double x = dadd(dadd(dadd(dmul(n0, M[0]), dmul(n1, M[3])), dmul(n2, M[6])), a.o);
            const double y = dadd(dadd(dadd(dmul(n0, M[1]), dmul(n1, M[4])), dmul(n2, M[7])), a.o);
            const double z = dadd(dadd(dadd(dmul(n0, M[2]), dmul(n1, M[5])), dmul(n2, M[8])), a.o);
            acc = __fadd_rn(acc, (float)interpolate(a.src, a.N, x, y, z, a.fill));
        }
        a.dst[i] = acc;
    }
}

// calculate_background, flag 0: per-block sums of the voxels outside the
// ellipsoid sum(((c - o) / h)^2) = 1, h = N / 2 (integer)
__global__ void background_sum_kernel(const float* m, int N, double o, double* part, long* cnt) {
    __shared__ double s[256];
    __shared__ long c[256];
    const long N3 = (long)N * N * N;
    const double h = (double)(N / 2);
    double acc = 0;
    long n = 0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N3; i += (long)gridDim.x * blockDim.x) {
        const long xx = i % N, yy = (i / N) % N, zz = i / ((long)N * N);
        double x2 = __ddiv_rn(dsub((double)xx, o), h), y2 = __ddiv_rn(dsub((double)yy, o), h),
               z2 = __ddiv_rn(dsub((double)zz, o), h);
        x2 = dmul(x2, x2);
        y2 = dmul(y2, y2);
        z2 = dmul(z2, z2);
        if (dsub(dadd(dadd(x2, y2), z2), 1.0) > 0) {
            acc = dadd(acc, (double)m[i]);
            ++n;
        }
    }
    s[threadIdx.x] = acc;
    c[threadIdx.x] = n;
    __syncthreads();
    for (int k = blockDim.x / 2; k; k >>= 1) {
        if ((int)threadIdx.x < k) {
            s[threadIdx.x] = dadd(s[threadIdx.x], s[threadIdx.x + k]);
            c[threadIdx.x] += c[threadIdx.x + k];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s[0];
        cnt[blockIdx.x] = c[0];
    }
}

// v * (1 / order), stored as float; then (trilinear maps) the sinc weight of
// filter_sinc (bsoft/src/img/Bimage_filter.cpp:484-509), stored as float
__global__ void scale_sinc_kernel(float* m, int N, double inv_order, int sinc) {
    const long NN = N, N3 = NN * NN * NN;
    const double o = (double)(N / 2);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N3; i += (long)gridDim.x * blockDim.x) {
        float v = (float)dmul((double)m[i], inv_order);
        if (sinc) {
            const long xx = i % NN, yy = (i / NN) % NN, zz = i / (NN * NN);
            const double dx = (xx - o) / N, dy = (yy - o) / N, dz = (zz - o) / N;
            const double rr = 3.14159265358979323846 * sqrt(dx * dx + dy * dy + dz * dz);
            if (rr != 0.0) {
                const double w = rr / sin(rr);
                v = (float)(w * w * v);
            }
        }
        m[i] = v;
    }
}

constexpr int BG_BLOCKS = 148 * 4;

// per-block sums of v and v^2 (Bimage::statistics of a real map)
__global__ void moments_kernel(const float* m, long n, double* s1, double* s2) {
    __shared__ double a[256], b[256];
    double x = 0, y = 0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double v = m[i];
        x = dadd(x, v);
        y = dadd(y, dmul(v, v));
    }
    a[threadIdx.x] = x;
    b[threadIdx.x] = y;
    __syncthreads();
    for (int k = blockDim.x / 2; k; k >>= 1) {
        if ((int)threadIdx.x < k) {
            a[threadIdx.x] = dadd(a[threadIdx.x], a[threadIdx.x + k]);
            b[threadIdx.x] = dadd(b[threadIdx.x], b[threadIdx.x + k]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        s1[blockIdx.x] = a[0];
        s2[blockIdx.x] = b[0];
    }
}

// Bimage::rescale (bsoft/src/img/Bimage_rescale.cpp:27-50): v scale + shift,
// stored as float; then the sinc weight
__global__ void rescale_sinc_kernel(float* m, int N, double scale, double shift, int sinc) {
    const long NN = N, N3 = NN * NN * NN;
    const double o = (double)(N / 2);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N3; i += (long)gridDim.x * blockDim.x) {
        float v = (float)dadd(dmul((double)m[i], scale), shift);
        if (sinc) {
            const long xx = i % NN, yy = (i / NN) % NN, zz = i / (NN * NN);
            const double dx = (xx - o) / N, dy = (yy - o) / N, dz = (zz - o) / N;
            const double rr = 3.14159265358979323846 * sqrt(dx * dx + dy * dy + dz * dz);
            if (rr != 0.0) {
                const double w = rr / sin(rr);
                v = (float)(w * w * v);
            }
        }
        m[i] = v;
    }
}

}  // namespace

// Matrix3(axis, angle) of the reference: the axis normalised (as Bsymmetry
// stores it, then again by Matrix3), a quaternion from the half angle, its
// matrix with entries below 1e-12 set to 0 and clamped to [-1, 1]
// (bsoft/include/Quaternion.h:34-41, bsoft/include/Matrix3.h:21-42).
static void normalize3(double v[3]) {
    const double ln = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (ln < 1e-30) { v[2] = 1.0; return; }
    const double d = 1.0 / ln;
    v[0] *= d; v[1] *= d; v[2] *= d;
}

void symmetrize_matrix(const double axis[3], double angle, double out[9]) {
    double u[3] = {axis[0], axis[1], axis[2]};
    normalize3(u);
    normalize3(u);
    const double a = angle / 2.0, sa = sin(a);
    double q[4] = {cos(a), u[0] * sa, u[1] * sa, u[2] * sa};
    for (double& v : q)
        if (fabs(v) < 1e-30) v = 0.0;
    const double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
    double d[9] = {q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3, 2 * q1 * q2 - 2 * q0 * q3, 2 * q1 * q3 + 2 * q0 * q2,
                   2 * q1 * q2 + 2 * q0 * q3, q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3, 2 * q2 * q3 - 2 * q0 * q1,
                   2 * q1 * q3 - 2 * q0 * q2, 2 * q2 * q3 + 2 * q0 * q1, q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3};
    for (int i = 0; i < 9; ++i) {
        double v = d[i];
        if (fabs(v) < 1e-12) v = 0.0;
        out[i] = v < -1.0 ? -1.0 : (v > 1.0 ? 1.0 : v);
    }
}

// The symmetrized map in place (buffer `map`, N^3 float; `tmp` the same
// size), then 1 / order and the sinc weight.
cudaError_t launch_symmetrize(const Context& c, float* map, float* tmp, bool sinc, cudaStream_t s) {
    const int N = c.g.map;
    const size_t nops = c.symz_orders.size();
    double* d_part = nullptr;
    long* d_cnt = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&d_part, sizeof(double) * BG_BLOCKS, s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_cnt, sizeof(long) * BG_BLOCKS, s);
    if (e != cudaSuccess) return e;
    background_sum_kernel<<<BG_BLOCKS, 256, 0, s>>>(map, N, (double)(N / 2), d_part, d_cnt);
    std::vector<double> part(BG_BLOCKS);
    std::vector<long> cnt(BG_BLOCKS);
    e = cudaMemcpyAsync(part.data(), d_part, sizeof(double) * BG_BLOCKS, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(long) * BG_BLOCKS, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(d_part, s);
    cudaFreeAsync(d_cnt, s);
    if (e != cudaSuccess) return e;
    double bkg = 0;
    long nm = 0;
    for (int i = 0; i < BG_BLOCKS; ++i) { bkg += part[i]; nm += cnt[i]; }
    const double fill = nm ? bkg / nm : 0.0;
    long order = 1;
    float* src = map;
    float* dst = tmp;
    for (size_t op = 0; op < nops; ++op) {
        const int k = c.symz_orders[op];
        order *= k;
        if (k < 2) continue;
        RotArgs a{};
        a.src = src; a.dst = dst; a.N = N; a.nrot = k - 1; a.o = (double)(N / 2); a.fill = fill;
        for (int j = 1; j < k; ++j)
            symmetrize_matrix(&c.symz_axes[3 * op], j * M_PI * 2.0 / k, a.m[j - 1]);
        rotate_sum_kernel<<<148 * 8, 256, 0, s>>>(a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        float* t = src; src = dst; dst = t;
    }
    if (src != map) {
        e = cudaMemcpyAsync(map, src, sizeof(float) * c.vol_elems(), cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return e;
    }
    scale_sinc_kernel<<<148 * 8, 256, 0, s>>>(map, N, order > 1 ? 1.0 / (double)order : 1.0, sinc ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace bsg

namespace bsg {

// Bimage::rescale_to_avg_std (bsoft/src/img/Bimage_rescale.cpp:163-182) of
// the real map in place, from its average and standard deviation
// (Bimage::statistics: sqrt(mean v^2 - mean^2)), then the sinc weight.
cudaError_t launch_rescale(const Context& c, float* map, double nuavg, double nustd, bool sinc, cudaStream_t s) {
    const int N = c.g.map;
    const long N3 = (long)c.vol_elems();
    double* d = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&d, sizeof(double) * 2 * BG_BLOCKS, s);
    if (e != cudaSuccess) return e;
    moments_kernel<<<BG_BLOCKS, 256, 0, s>>>(map, N3, d, d + BG_BLOCKS);
    std::vector<double> h(2 * BG_BLOCKS);
    e = cudaMemcpyAsync(h.data(), d, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(d, s);
    if (e != cudaSuccess) return e;
    double s1 = 0, s2 = 0;
    for (int i = 0; i < BG_BLOCKS; ++i) { s1 += h[i]; s2 += h[BG_BLOCKS + i]; }
    const double avg = s1 / N3;
    double sd = s2 / N3 - avg * avg;
    sd = sd > 0 ? sqrt(sd) : 0.0;
    const double scale = sd > 1e-30 ? nustd / sd : 1.0, shift = nuavg - avg * scale;
    rescale_sinc_kernel<<<148 * 8, 256, 0, s>>>(map, N, scale, shift, sinc ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace bsg
