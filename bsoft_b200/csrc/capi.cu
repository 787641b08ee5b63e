// capi.cu - the extern "C" boundary of libbsgpu.so (declared in
// include/bsgpu.h): context lifetime, device memory, the batched insertion
// pipeline (image upload, 2-D stage, gridding) and map finishing.
#include "context.cuh"
#include "fft_dev.cuh"
#include "lattice.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <vector>

namespace bsg {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

cudaError_t prepare_fft2d_attributes();
cudaError_t prepare_finish_attributes();
cudaError_t launch_weigh(const Context& c, int imap, cudaStream_t s);
cudaError_t launch_ifft3(const Context& c, float2* vol, float* real_out, bool sinc, cudaStream_t s);
int insert_num_shapes();
void insert_shape(int i, int* tx, int* ty, int* tz);
cudaError_t prepare_insert_attributes();
cudaError_t launch_map_sums(double2* dv, double* dw, const double2* vol, const double* w, const double2* e,
                            const double* ew, int N, int zsplit, cudaStream_t s);

struct Timed {
    cudaEvent_t a, b;
    int kind;   // 0 insert, 1 fft2d, 2 h2d
};

// Batches alternate between two sets of buffers (buf = seq & 1).  Three
// streams: copy_stream uploads batch i's images, fft_stream runs batch i's
// 2-D transforms and `stream` grids batch i - 1.  The transforms' blocks
// are dispatched once the gridding kernel has dispatched all of its own, so
// they fill the SMs its last (lightest) tiles leave idle.  (At high stream
// priority they displace gridding blocks instead and the step is slower.)
// Gridding stays in batch order on `stream`: the accumulation order does
// not change.
struct Recon : Context {
    cudaStream_t copy_stream = nullptr;
    cudaStream_t fft_stream = nullptr;
    float* d_imgbuf[2] = {nullptr, nullptr};
    DevParticle* h_partbuf[2] = {nullptr, nullptr};
    DevParticle* d_partbuf[2] = {nullptr, nullptr};
    DevParticle* d_psymbuf[2] = {nullptr, nullptr};
    size_t psymbuf_cap[2] = {0, 0};
    float2* d_specbuf[2] = {nullptr, nullptr};
    cudaEvent_t copy_done[2] = {nullptr, nullptr};
    cudaEvent_t fft_done[2] = {nullptr, nullptr};       // batch's spectra written
    cudaEvent_t compute_done[2] = {nullptr, nullptr};   // batch gridded: its buffers are free
    std::vector<Timed> timed;
    bool broken = false;
    long seq = 0;                    // batches issued over the context's life (staging buffer = seq & 1)
    long nexp = 0;                   // expanded gridding records of the current batch (0: none)
};

static bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

static int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(BSG_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

static void host_twiddles(int L, std::vector<float2>& out) {
    out.resize(std::max(1, L / 2));
    for (int j = 0; j < L / 2; ++j) {
        double a = -2.0 * M_PI * j / L;
        out[j] = make_float2((float)cos(a), (float)sin(a));
    }
    if (L / 2 == 0) out[0] = make_float2(1.f, 0.f);
}

// 32-double C-ABI record -> device record (see bsgpu.h for the layout)
// ewh: the Ewald surface's +-lambda/2 for this record (0: the plane)
static void make_dev_particle(const Recon& r, const double* q, DevParticle& d, double ewh = 0.0) {
    const Geometry& g = r.g;
    memset(&d, 0, sizeof(d));
    d.shx = q[0] / g.ft * 2.0 * M_PI;                 // Bimage_complex.cpp:510 shift = origin/size*2pi
    d.shy = q[1] / g.ft * 2.0 * M_PI;
    d.bx = q[2];
    d.by = q[3];
    const double* R = q + 4;
    const double pixel = q[13], scale = q[14] > 0 ? q[14] : 1.0;
    d.fs = 1.0 / (g.ft * pixel);                       // mg_ctf.cpp:84 freq_scale = 1/real_size
    d.c00 = q[16]; d.c20 = q[17]; d.c22 = q[18]; d.c2m2 = q[19]; d.c40 = q[20]; d.c11 = q[21]; d.c1m1 = q[22];
    const double inv = scale / (g.ft * pixel);         // Bimage_reconstruct.cpp:145 invscale
    for (int i = 0; i < 3; ++i) {
        d.ad[i] = R[3 * i + 0] * inv * g.mscale;
        d.bd[i] = R[3 * i + 1] * inv * g.mscale;
        d.af[i] = (float)d.ad[i];
        d.bf[i] = (float)d.bd[i];
    }
    for (int i = 0; i < 3; ++i) d.cd[i] = R[3 * i + 2] * g.mscale;
    for (int i = 0; i < 3; ++i) {
        d.iad[i] = fabs(d.ad[i]) > 1e-12 ? 1.0 / d.ad[i] : 0.0;
        d.ibd[i] = fabs(d.bd[i]) > 1e-12 ? 1.0 / d.bd[i] : 0.0;
    }
    d.inv = inv;
    double nn = sqrt(R[2] * R[2] + R[5] * R[5] + R[8] * R[8]);
    if (nn <= 0) nn = 1;
    d.nrm[0] = R[2] / nn; d.nrm[1] = R[5] / nn; d.nrm[2] = R[8] / nn;
    d.slab = (float)(fabs(d.nrm[0]) + fabs(d.nrm[1]) + fabs(d.nrm[2]));
    d.step = (float)(inv * g.mscale);
    d.inv2 = inv * inv;
    d.inv_st2 = 1.0 / ((double)d.step * (double)d.step);
    d.inv_step = 1.0f / d.step;
    for (int i = 0; i < 3; ++i) d.ib[i] = fabsf(d.bf[i]) > 1e-6f ? 1.0f / d.bf[i] : 0.0f;
    double pw = q[15];
    double pad_ratio = (double)g.ft / (double)g.n;     // mg_reconstruct.cpp:192-199
    if (pad_ratio > 1) { pad_ratio *= pad_ratio * 0.6; pw /= pad_ratio; }
    d.pw = (float)pw;
    d.half = (int)q[23];
    // the curvature bound ewh inv2 mscale |p + q| <= ewh inv2 mscale ft sqrt(2)
    // per pixel step of a lattice vector, and the surface's largest offset
    d.ewh = ewh;
    const double hf = g.ft / 2.0;
    d.ezmax = (float)(fabs(d.ewh) * 2.0 * hf * hf * d.inv2 * g.mscale * 1.0001);
    const double curve = fabs(d.ewh) * d.inv2 * g.mscale * g.ft * 1.4142135623730951 * 1.0001;
    d.lat = pack_lattice(choose_lattice(d.ad, d.bd, 16, curve));
    // particle_reconstruct's rescale_to_avg_std(0, 1) under -rescale
    // (mg_reconstruct.cpp:155): v * scale + shift, scale 0 = none
    d.na = q[24] != 0 ? q[24] : 1.0;
    d.nb = q[24] != 0 ? q[25] : 0.0;
}

static bool needs_gate(const Recon& r, const DevParticle* parts, long np) {
    const double hf = r.g.ft / 2.0;
    for (long i = 0; i < np; ++i) {
        const double s2max = 2.0 * hf * hf * parts[i].inv2;
        if (s2max > r.g.maxs2) return true;
        if ((r.g.maxs2 - s2max) * r.g.mscale < 1.0) return true;
        if (r.g.mins2 > 0) return true;
    }
    return false;
}

// Half-space gridding (insert.cu, walk_edges) applies to trilinear
// insertion of planes without the FOM channels; the split is the first
// multiple of 8 above N/2, a tile boundary for every shape.  0: full map.
static int half_space_split(const Recon& r) {
    if (!r.half_space || r.ewald_seen || r.g.interp != 2 || r.g.fom) return 0;
    const int N = r.g.map, z = (N / 2 / 8 + 1) * 8;
    return z < N ? z : 0;
}

// Tile visiting order for the current shape: nearest to the Fourier origin
// (counting wrap-around) first, since every particle's plane passes there;
// with half-space gridding the tiles above the split, which grid only the
// unpaired pixels, come last.
static int set_shape(Recon* r, int shape) {
    if (shape < 0 || shape >= insert_num_shapes()) return fail(BSG_ERR_ARG, "tile shape %d out of range", shape);
    // in-flight gridding reads the tile order and the replica buffers
    CK(cudaStreamSynchronize(r->stream));
    int tx, ty, tz;
    insert_shape(shape, &tx, &ty, &tz);
    const int N = r->g.map;
    const int zs = r->zsplit;
    const int nx = (N + tx - 1) / tx, ny = (N + ty - 1) / ty, nz = (N + tz - 1) / tz;
    std::vector<std::pair<double, int>> d((size_t)nx * ny * nz);
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                auto dist = [N](double c) { return std::min(fabs(c), fabs(c - N)); };
                const double cx = dist((x + 0.5) * tx), cy = dist((y + 0.5) * ty), cz = dist((z + 0.5) * tz);
                const int i = (z * ny + y) * nx + x;
                const double last = (zs > 0 && z * tz >= zs) ? 4.0 * N * N : 0.0;
                d[i] = {last + cx * cx + cy * cy + cz * cz, i};
            }
    std::stable_sort(d.begin(), d.end());
    std::vector<int> order(d.size());
    for (size_t i = 0; i < d.size(); ++i) order[i] = d[i].second;
    CK(cudaMemcpy(r->d_tile_order, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice));
    r->shape = shape;
    // replicas: enough warps to fill the GPU several times over and to split
    // the tiles near the origin, which every particle reaches (at 256^3 two
    // replicas measured 2.5% faster than four, and halve the partial sums)
    const long ntiles = (long)nx * ny * nz;
    int R = (int)std::min<long>(16, std::max<long>(2, (65536 + ntiles - 1) / ntiles));
    const size_t need = (size_t)R * (r->g.fom ? 5 : 3) * r->vol_elems() * sizeof(double);
    if (r->d_part_sums) { cudaFree(r->d_part_sums); r->d_part_sums = nullptr; }
    if (cudaMalloc((void**)&r->d_part_sums, need) != cudaSuccess) {
        // not enough memory for replicas: run each tile in one warp
        r->d_part_sums = nullptr;
        R = 1;
    }
    r->replicas = R;
    return BSG_OK;
}

// Switch half-space gridding on or off.  Off: the accumulators become the
// full map's sums (read_sums, in place).  On: only while they are empty (a
// full map's sums cannot be split into paired and unpaired parts).
static int set_half_space(Recon* r, bool on) {
    const int old = r->zsplit;
    const bool was = r->half_space;
    r->half_space = on;
    const int z = half_space_split(*r);
    if (z == old) return BSG_OK;
    const int N = r->g.map;
    if (z > 0 && r->dirty) {
        r->half_space = was;
        return fail(BSG_ERR_STATE, "half-space gridding can be switched on only with empty accumulators "
                                   "(before inserting, or after bsg_recon_reset)");
    }
    CK(cudaStreamSynchronize(r->stream));
    auto free_e = [r]() {
        for (int i = 0; i < 2; ++i) {
            if (r->d_evol[i]) cudaFree(r->d_evol[i]);
            if (r->d_ew[i]) cudaFree(r->d_ew[i]);
            r->d_evol[i] = nullptr;
            r->d_ew[i] = nullptr;
        }
    };
    if (old > 0) {
        for (int i = 0; i < r->nhalves; ++i)
            CK(launch_map_sums(r->d_vol[i], r->d_w[i], r->d_vol[i], r->d_w[i], r->d_evol[i], r->d_ew[i], N, old,
                               r->stream));
        CK(cudaStreamSynchronize(r->stream));
        free_e();
    }
    r->zsplit = 0;
    if (z > 0) {
        const size_t n = (size_t)z * N * N;
        for (int i = 0; i < r->nhalves; ++i) {
            if (cudaMalloc((void**)&r->d_evol[i], sizeof(double2) * n) != cudaSuccess ||
                cudaMalloc((void**)&r->d_ew[i], sizeof(double) * n) != cudaSuccess) {
                // not enough memory for the unpaired sums: the full map
                cudaGetLastError();
                free_e();
                r->half_space = false;
                return set_shape(r, r->shape);
            }
            CK(cudaMemsetAsync(r->d_evol[i], 0, sizeof(double2) * n, r->stream));
            CK(cudaMemsetAsync(r->d_ew[i], 0, sizeof(double) * n, r->stream));
        }
        r->zsplit = z;
    }
    return set_shape(r, r->shape);
}

// Failures the kernels report through the mapped status word (bounded waits).
static int check_status(Recon* r) {
    if (r->h_status && *(volatile int*)r->h_status) {
        r->broken = true;
        return fail(BSG_ERR_CUDA, "a gridding kernel gave up waiting for a shared-memory tile; results are invalid");
    }
    return BSG_OK;
}

static int alloc(void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return fail(BSG_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    return BSG_OK;
}

static void free_all(Recon* r) {
    auto F = [](void* p) { if (p) cudaFree(p); };
    for (int i = 0; i < 2; ++i) {
        F(r->d_imgbuf[i]); F(r->d_vol[i]); F(r->d_w[i]); F(r->d_pow[i]); F(r->d_w2[i]);
        F(r->d_evol[i]); F(r->d_ew[i]);
        F(r->d_half_weighed[i]);
        F(r->d_partbuf[i]); F(r->d_psymbuf[i]); F(r->d_specbuf[i]);
        if (r->h_partbuf[i]) cudaFreeHost(r->h_partbuf[i]);
        if (r->copy_done[i]) cudaEventDestroy(r->copy_done[i]);
        if (r->fft_done[i]) cudaEventDestroy(r->fft_done[i]);
        if (r->compute_done[i]) cudaEventDestroy(r->compute_done[i]);
    }
    F(r->d_bkg); F(r->d_phase); F(r->d_rows); F(r->d_tw); F(r->d_twmap);
    F(r->d_work); F(r->d_map); F(r->d_fom); F(r->d_fsc); F(r->d_tile_order); F(r->d_part_sums); F(r->d_symtmp);
    if (r->h_status) cudaFreeHost(r->h_status);
    for (auto& t : r->timed) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
    r->timed.clear();
    if (r->stream) cudaStreamDestroy(r->stream);
    if (r->copy_stream) cudaStreamDestroy(r->copy_stream);
    if (r->fft_stream) cudaStreamDestroy(r->fft_stream);
}

// The batch's 2-D transforms on fft_stream into the spectra buffer `buf`,
// then (insert) its gridding on `stream` once they are done.
static int run_batch_kernels(Recon* r, int buf, const float* d_img, long np, bool insert) {
    cudaStream_t f = r->fft_stream, s = r->stream;
    float2* spec_out = r->d_specbuf[buf];
    cudaEvent_t a = nullptr, b = nullptr;
    // the spectra buffer is free once the batch two back has been gridded
    CK(cudaStreamWaitEvent(f, r->compute_done[buf], 0));
    if (r->timing) { cudaEventCreate(&a); cudaEventCreate(&b); cudaEventRecord(a, f); }
    CK(launch_background(*r, d_img, (int)np, f));
    CK(launch_rows(*r, d_img, (int)np, f));
    CK(launch_cols(*r, (int)np, spec_out, f));
    r->stats.launches += 3;
    if (r->timing) { cudaEventRecord(b, f); r->timed.push_back({a, b, 1}); }
    CK(cudaEventRecord(r->fft_done[buf], f));
    CK(cudaStreamWaitEvent(s, r->fft_done[buf], 0));
    if (!insert) return BSG_OK;
    for (int h = 0; h < r->nhalves; ++h) {
        if (r->timing) { cudaEventCreate(&a); cudaEventCreate(&b); cudaEventRecord(a, s); }
        if (r->nexp > 0) CK(launch_insert(*r, spec_out, r->d_psym, (int)r->nexp, r->nhalves == 2 ? h : -1, s));
        else CK(launch_insert(*r, spec_out, r->d_part, (int)np, r->nhalves == 2 ? h : -1, s));
        if (r->timing) { cudaEventRecord(b, s); r->timed.push_back({a, b, 0}); }
        r->stats.launches += r->replicas > 1 ? 2 : 1;     // gridding (+ replica combine)
        r->stats.insert_launches += 1;
    }
    r->stats.particles += np;
    return BSG_OK;
}

// Upload one batch's particle records through a pinned staging buffer.
static int upload_params(Recon* r, int buf, const double* params, long np) {
    // the staging buffer may still feed an in-flight copy from two batches ago
    CK(cudaEventSynchronize(r->compute_done[buf]));
    DevParticle* hp = r->h_partbuf[buf];
    for (long i = 0; i < np; ++i) {
        make_dev_particle(*r, params + i * BSG_PARTICLE_DOUBLES, hp[i]);
        hp[i].spec = (int)i;
    }
    r->g.gate = needs_gate(*r, hp, np) ? 1 : 0;
    // half-space gridding: the unpaired pixels (row or column -ft/2) lie at
    // least ft/2 pixel steps from the origin, and no pixel lies beyond the
    // transform's corner, ft/2 sqrt(2) steps
    {
        double smin = 1e300, smax = 0;
        for (long i = 0; i < np; ++i) {
            smin = std::min(smin, (double)hp[i].step);
            smax = std::max(smax, (double)hp[i].step);
        }
        const double hf = r->g.ft / 2.0;
        r->edge_rmin = np ? hf * smin * (1.0 - 1e-6) - 1e-3 : 0.0;
        r->edge_rmax = hf * smax * 1.4142136 * (1.0 + 1e-6) + 2.0;
    }
    r->d_part = r->d_partbuf[buf];
    CK(cudaMemcpyAsync(r->d_part, hp, sizeof(DevParticle) * np, cudaMemcpyHostToDevice, r->fft_stream));
    const long nsym = std::max(1L, (long)r->sym.size() / 9);
    bool ewald = false;
    for (long i = 0; i < np && !ewald; ++i) ewald = params[i * BSG_PARTICLE_DOUBLES + 26] != 0;
    r->nexp = 0;
    r->g.ewald = ewald ? 1 : 0;
    if (nsym > 1 || ewald) {
        // one gridding record per (particle, operator): matrix S R, the
        // particle's spectrum (fspace_pack_2D(p, View, sym, ...),
        // Bimage_reconstruct.cpp:248-266)
        const size_t need = (size_t)np * nsym * (ewald ? 2 : 1);
        if (need > r->psymbuf_cap[buf]) {
            if (r->d_psymbuf[buf]) cudaFree(r->d_psymbuf[buf]);
            r->d_psymbuf[buf] = nullptr;
            r->psymbuf_cap[buf] = 0;
            CK(cudaMalloc((void**)&r->d_psymbuf[buf], sizeof(DevParticle) * need));
            r->psymbuf_cap[buf] = need;
        }
        r->d_psym = r->d_psymbuf[buf];
        // pageable staging: cudaMemcpyAsync has copied it when it returns,
        // and the device buffer is rewritten in stream order
        r->h_psym.resize(need);
        double q[BSG_PARTICLE_DOUBLES];
        size_t k = 0;
        for (long i = 0; i < np; ++i) {
            const double* p0 = params + i * BSG_PARTICLE_DOUBLES;
            // Ewald sphere (fspace_pack_2D with ewald_wavelength = lambda,
            // Bimage_reconstruct.cpp:157-168): both surfaces s_z = +-(lambda/2) s^2
            const double lam = p0[26];
            const int nsurf = lam != 0 ? 2 : 1;
            for (long s = 0; s < nsym; ++s) {
                memcpy(q, p0, sizeof(q));
                if (nsym > 1) {
                    const double* S = &r->sym[9 * s];
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < 3; ++b)
                            q[4 + 3 * a + b] = S[3 * a + 0] * p0[4 + 0 * 3 + b] + S[3 * a + 1] * p0[4 + 1 * 3 + b] +
                                               S[3 * a + 2] * p0[4 + 2 * 3 + b];
                }
                for (int t = 0; t < nsurf; ++t) {
                    DevParticle& d = r->h_psym[k++];
                    make_dev_particle(*r, q, d, nsurf == 2 ? (t == 0 ? lam / 2 : -(lam / 2)) : 0.0);
                    d.spec = (int)i;
                }
            }
        }
        r->nexp = (long)k;
        CK(cudaMemcpyAsync(r->d_psym, r->h_psym.data(), sizeof(DevParticle) * k, cudaMemcpyHostToDevice,
                           r->fft_stream));
    }
    return BSG_OK;
}

static int process(Recon* r, const float* images, const double* params, long nparts, int flags,
                   float* spectra_out) {
    const size_t img_elems = (size_t)r->g.n * r->g.n;
    const bool dev = flags & BSG_DEVICE_PTR;
    for (long off = 0; off < nparts; off += r->batch) {
        const long np = std::min<long>(r->batch, nparts - off);
        // alternate the staging buffers across calls too, so that one call's
        // upload overlaps the previous call's kernels
        const int buf = (int)(r->seq++ & 1);
        int rc = upload_params(r, buf, params + off * BSG_PARTICLE_DOUBLES, np);
        if (rc) return rc;
        if (!spectra_out && r->g.ewald && !r->ewald_seen) {
            // an Ewald surface is not Hermitian: the full map from here on
            r->ewald_seen = true;
            rc = set_half_space(r, r->half_space);
            if (rc) return rc;
        }
        if (!spectra_out) r->dirty = true;
        const float* d_img;
        if (dev) {
            d_img = images + off * img_elems;
        } else {
            // the buffer is free once the batch that last used it has finished
            CK(cudaStreamWaitEvent(r->copy_stream, r->compute_done[buf], 0));
            cudaEvent_t a = nullptr, b = nullptr;
            if (r->timing) { cudaEventCreate(&a); cudaEventCreate(&b); cudaEventRecord(a, r->copy_stream); }
            CK(cudaMemcpyAsync(r->d_imgbuf[buf], images + off * img_elems, sizeof(float) * img_elems * np,
                               cudaMemcpyHostToDevice, r->copy_stream));
            if (r->timing) { cudaEventRecord(b, r->copy_stream); r->timed.push_back({a, b, 2}); }
            CK(cudaEventRecord(r->copy_done[buf], r->copy_stream));
            CK(cudaStreamWaitEvent(r->fft_stream, r->copy_done[buf], 0));
            d_img = r->d_imgbuf[buf];
        }
        r->d_spec = r->d_specbuf[buf];
        rc = run_batch_kernels(r, buf, d_img, np, spectra_out == nullptr);
        if (rc) return rc;
        if (spectra_out) {
            // centred device layout -> the reference's pixel order (the four
            // quadrants swap places)
            const int ft = r->g.ft, hf = ft / 2;
            const size_t sp = sizeof(float2) * r->spec_pitch(), dp = sizeof(float2) * ft;
            const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
            for (long i = 0; i < np; ++i) {
                const float2* src = r->d_spec + (size_t)i * r->spec_elems();
                float2* dst = reinterpret_cast<float2*>(spectra_out) + (size_t)(off + i) * ft * ft;
                for (int qy = 0; qy < 2; ++qy)
                    for (int qx = 0; qx < 2; ++qx) {
                        // reference rows [qy*hf, qy*hf+hf) hold k = qy ? rows - ft : rows
                        const float2* s0 = src + (size_t)(qy ? 0 : hf) * r->spec_pitch() + (qx ? 0 : hf);
                        float2* d0 = dst + (size_t)qy * hf * ft + qx * hf;
                        CK(cudaMemcpy2DAsync(d0, dp, s0, sp, sizeof(float2) * hf, hf, kind, r->stream));
                    }
            }
        }
        CK(cudaEventRecord(r->compute_done[buf], r->stream));
    }
    return BSG_OK;
}

static int ensure_finish_buffers(Recon* r) {
    const size_t N3 = r->vol_elems();
    if (!r->d_work) { int rc = alloc((void**)&r->d_work, sizeof(float2) * N3); if (rc) return rc; }
    if (!r->d_map) { int rc = alloc((void**)&r->d_map, sizeof(float) * N3); if (rc) return rc; }
    if (r->g.fom && !r->d_fom) { int rc = alloc((void**)&r->d_fom, sizeof(float) * N3); if (rc) return rc; }
    return BSG_OK;
}

}  // namespace bsg

using namespace bsg;

extern "C" {

const char* bsg_last_error(void) { return g_err; }
const char* bsg_version(void) { return "bsgpu 0.1.0 (sm_100a)"; }

int bsg_recon_create(const bsg_recon_config* cfg, bsg_recon** out) {
    if (!cfg || !out) return fail(BSG_ERR_ARG, "bsg_recon_create: null argument");
    *out = nullptr;
    const int n = cfg->n, ft = cfg->ft, N = cfg->map;
    if (n < 2 || !is_pow2(ft) || ft < 32 || ft > 1024 || ft < n)
        return fail(BSG_ERR_ARG, "bsg_recon_create: transform size %d must be a power of two in [32, 1024] and >= box %d", ft, n);
    int radices[16];
    if ((N & 1) || N < 8 || N > 512 || N > ft || factor_radices(N, radices) < 0)
        return fail(BSG_ERR_ARG, "bsg_recon_create: map size %d must be even, in [8, 512], <= %d and a product of 2, 3, 5, 7", N, ft);
    if (cfg->interp < 0 || cfg->interp > 2) return fail(BSG_ERR_ARG, "bsg_recon_create: interp %d", cfg->interp);
    if (cfg->nmaps < 1 || cfg->nmaps > 3) return fail(BSG_ERR_ARG, "bsg_recon_create: nmaps %d", cfg->nmaps);
    if (!(cfg->map_sampling > 0) || !(cfg->hi_res > 0)) return fail(BSG_ERR_ARG, "bsg_recon_create: sampling/resolution");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device || cfg->device < 0)
        return fail(BSG_ERR_NODEV, "bsg_recon_create: CUDA device %d not available", cfg->device);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess || prop.major < 10)
        return fail(BSG_ERR_NODEV, "bsg_recon_create: device %d is not sm_100 class", cfg->device);
    CK(cudaSetDevice(cfg->device));

    Recon* r = new (std::nothrow) Recon();
    if (!r) return fail(BSG_ERR_NOMEM, "bsg_recon_create: host allocation");
    r->cfg = *cfg;
    r->device = cfg->device;
    Geometry& g = r->g;
    g.n = n; g.ft = ft; g.map = N; g.logft = ilog2i(ft);
    g.interp = cfg->interp; g.ctf_action = cfg->ctf_action; g.wiener = cfg->wiener;
    g.hi_res = cfg->hi_res < 0.5 ? 0.5 : cfg->hi_res;      // Bimage_reconstruct.cpp:136
    g.maxs2 = 1.0 / (g.hi_res * g.hi_res);
    g.mins2 = 0.0;
    g.ctf_shi2 = 1.0 / (cfg->hi_res * cfg->hi_res);        // mg_ctf.cpp:50-58
    g.mscale = N * cfg->map_sampling;
    g.fom = cfg->fom ? 1 : 0;
    g.gate = 1;
    r->nhalves = cfg->nmaps >= 2 ? 2 : 1;
    int batch = cfg->batch;
    if (batch <= 0) {
        const double per = 8.0 * ft * ft;
        batch = (int)std::min(4096.0, std::max(32.0, 2.0e9 / per));
    }
    r->batch = batch;

    int rc = BSG_OK;
    auto A = [&](void** p, size_t bytes) { if (!rc) rc = alloc(p, bytes); };
    if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&r->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&r->fft_stream, cudaStreamNonBlocking) != cudaSuccess) {
        free_all(r); delete r;
        return fail(BSG_ERR_CUDA, "bsg_recon_create: stream creation failed");
    }
    const size_t N3 = (size_t)N * N * N;
    for (int i = 0; i < 2; ++i) {
        A((void**)&r->d_imgbuf[i], sizeof(float) * (size_t)n * n * batch);
        if (!rc && cudaMallocHost((void**)&r->h_partbuf[i], sizeof(DevParticle) * batch) != cudaSuccess)
            rc = fail(BSG_ERR_NOMEM, "bsg_recon_create: pinned host allocation");
        A((void**)&r->d_partbuf[i], sizeof(DevParticle) * batch);
        A((void**)&r->d_specbuf[i], sizeof(float2) * (size_t)(ft + 1) * (ft + 2) * batch);
        if (!rc && cudaMemset(r->d_specbuf[i], 0, sizeof(float2) * (size_t)(ft + 1) * (ft + 2) * batch) != cudaSuccess)
            rc = fail(BSG_ERR_CUDA, "bsg_recon_create: clearing the spectra buffer");
        if (!rc && (cudaEventCreateWithFlags(&r->copy_done[i], cudaEventDisableTiming) != cudaSuccess ||
                    cudaEventCreateWithFlags(&r->fft_done[i], cudaEventDisableTiming) != cudaSuccess ||
                    cudaEventCreateWithFlags(&r->compute_done[i], cudaEventDisableTiming) != cudaSuccess))
            rc = fail(BSG_ERR_CUDA, "bsg_recon_create: event creation failed");
    }
    A((void**)&r->d_bkg, sizeof(double) * batch);
    A((void**)&r->d_phase, sizeof(float2) * 2 * ft * (size_t)batch);
    A((void**)&r->d_rows, sizeof(float2) * (size_t)n * (ft / 2 + 1) * batch);
    A((void**)&r->d_tw, sizeof(float2) * std::max(1, ft / 2));
    A((void**)&r->d_twmap, sizeof(float2) * N);
    for (int h = 0; h < r->nhalves; ++h) {
        A((void**)&r->d_vol[h], sizeof(double2) * N3);
        A((void**)&r->d_w[h], sizeof(double) * N3);
        if (g.fom) { A((void**)&r->d_pow[h], sizeof(double) * N3); A((void**)&r->d_w2[h], sizeof(double) * N3); }
    }
    if (!rc && cudaHostAlloc((void**)&r->h_status, sizeof(int), cudaHostAllocMapped) != cudaSuccess)
        rc = fail(BSG_ERR_NOMEM, "bsg_recon_create: mapped status word");
    if (!rc && cudaHostGetDevicePointer((void**)&r->d_status, r->h_status, 0) != cudaSuccess)
        rc = fail(BSG_ERR_CUDA, "bsg_recon_create: status word mapping");
    if (!rc) *r->h_status = 0;
    if (!rc) rc = alloc((void**)&r->d_tile_order, sizeof(int) * (size_t)((N + 7) / 8) * ((N + 7) / 8) * ((N + 7) / 8));
    if (rc) { free_all(r); delete r; return rc; }
    std::vector<float2> tw;
    host_twiddles(ft, tw);
    cudaError_t e = cudaMemcpy(r->d_tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice);
    tw.resize(N);
    for (int j = 0; j < N; ++j) {
        const double ang = -2.0 * M_PI * j / N;
        tw[j] = make_float2((float)cos(ang), (float)sin(ang));
    }
    if (e == cudaSuccess) e = cudaMemcpy(r->d_twmap, tw.data(), sizeof(float2) * N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = prepare_fft2d_attributes();
    if (e == cudaSuccess) e = prepare_finish_attributes();
    if (e == cudaSuccess) e = prepare_insert_attributes();
    if (e != cudaSuccess) { free_all(r); delete r; return fail(BSG_ERR_CUDA, "bsg_recon_create: %s", cudaGetErrorString(e)); }
    for (int i = 0; i < 2; ++i) {
        cudaEventRecord(r->compute_done[i], r->stream);
    }
    {
        r->shape = 0;
        r->zsplit = 0;
        const int rc2 = half_space_split(*r) > 0 ? set_half_space(r, true) : set_shape(r, 0);
        if (rc2) { free_all(r); delete r; return rc2; }
    }
    *out = reinterpret_cast<bsg_recon*>(r);
    return bsg_recon_reset(*out);
}

void bsg_recon_destroy(bsg_recon* h) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r) return;
    cudaSetDevice(r->device);
    if (r->stream) cudaStreamSynchronize(r->stream);
    if (r->fft_stream) cudaStreamSynchronize(r->fft_stream);
    if (r->copy_stream) cudaStreamSynchronize(r->copy_stream);
    free_all(r);
    delete r;
}

int bsg_recon_reset(bsg_recon* h) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r) return fail(BSG_ERR_ARG, "bsg_recon_reset: null context");
    CK(cudaSetDevice(r->device));
    const size_t N3 = r->vol_elems();
    for (int i = 0; i < r->nhalves; ++i) {
        CK(cudaMemsetAsync(r->d_vol[i], 0, sizeof(double2) * N3, r->stream));
        CK(cudaMemsetAsync(r->d_w[i], 0, sizeof(double) * N3, r->stream));
        if (r->zsplit > 0) {
            const size_t n = (size_t)r->zsplit * r->g.map * r->g.map;
            CK(cudaMemsetAsync(r->d_evol[i], 0, sizeof(double2) * n, r->stream));
            CK(cudaMemsetAsync(r->d_ew[i], 0, sizeof(double) * n, r->stream));
        }
        if (r->g.fom) {
            CK(cudaMemsetAsync(r->d_pow[i], 0, sizeof(double) * N3, r->stream));
            CK(cudaMemsetAsync(r->d_w2[i], 0, sizeof(double) * N3, r->stream));
        }
    }
    r->dirty = false;
    return BSG_OK;
}

int bsg_recon_insert(bsg_recon* h, const float* images, const double* params, long nparts, int flags) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || !images || !params || nparts < 0) return fail(BSG_ERR_ARG, "bsg_recon_insert: bad argument");
    if (r->broken) return fail(BSG_ERR_STATE, "bsg_recon_insert: context unusable after an earlier CUDA error");
    if (nparts == 0) return BSG_OK;
    for (long i = 0; i < nparts; ++i) {
        const double* q = params + i * BSG_PARTICLE_DOUBLES;
        if (!(q[13] > 0)) return fail(BSG_ERR_ARG, "bsg_recon_insert: particle %ld has pixel size %g", i, q[13]);
        const int half = (int)q[23];
        if (half < 0 || half > 1) return fail(BSG_ERR_ARG, "bsg_recon_insert: particle %ld half-map index %d", i, half);
    }
    CK(cudaSetDevice(r->device));
    int rc = process(r, images, params, nparts, flags, nullptr);
    if (rc == BSG_ERR_CUDA) r->broken = true;
    return rc;
}

int bsg_particle_spectra(bsg_recon* h, const float* images, const double* params, long nparts, float* out, int flags) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || !images || !params || !out || nparts < 0) return fail(BSG_ERR_ARG, "bsg_particle_spectra: bad argument");
    CK(cudaSetDevice(r->device));
    int rc = process(r, images, params, nparts, flags, out);
    if (rc) return rc;
    CK(cudaStreamSynchronize(r->stream));
    return BSG_OK;
}

int bsg_recon_finish(bsg_recon* h, int imap, float* map_out, float* fom_out, int flags) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || !map_out) return fail(BSG_ERR_ARG, "bsg_recon_finish: bad argument");
    if (imap < 0 || imap > 2 || (imap > 0 && r->nhalves < 2))
        return fail(BSG_ERR_ARG, "bsg_recon_finish: map %d not available (nmaps = %d)", imap, r->cfg.nmaps);
    if (fom_out && !r->g.fom) return fail(BSG_ERR_ARG, "bsg_recon_finish: FOM requested but fom = 0");
    CK(cudaSetDevice(r->device));
    int rc = ensure_finish_buffers(r);
    if (rc) return rc;
    const bool sinc = (flags & BSG_SINC) != 0;
    const bool dev = (flags & BSG_DEVICE_PTR) != 0;
    float* dst = dev ? map_out : r->d_map;
    const bool symz = !r->symz_orders.empty(), resc = r->rescale_std > 0;
    CK(launch_weigh(*r, imap, r->stream));
    // with symmetrization after reconstruction (mode 1) and rescaling, the
    // sinc weight follows them, as breconstruct applies filter_sinc to the
    // written map (breconstruct.cpp:332-346, 360)
    CK(launch_ifft3(*r, r->d_work, dst, sinc && !symz && !resc, r->stream));
    r->stats.launches += 4;
    if (symz) {
        if (!r->d_symtmp) {
            int rc = alloc((void**)&r->d_symtmp, sizeof(float) * r->vol_elems());
            if (rc) return rc;
        }
        CK(launch_symmetrize(*r, dst, r->d_symtmp, sinc && !resc, r->stream));
        long ops = 0;
        for (int k : r->symz_orders) ops += k > 1;
        r->stats.launches += 2 + ops;
    }
    if (resc) {
        CK(launch_rescale(*r, dst, r->rescale_avg, r->rescale_std, sinc, r->stream));
        r->stats.launches += 2;
    }
    const size_t N3 = r->vol_elems();
    if (!dev) CK(cudaMemcpyAsync(map_out, r->d_map, sizeof(float) * N3, cudaMemcpyDeviceToHost, r->stream));
    if (fom_out) CK(cudaMemcpyAsync(fom_out, r->d_fom, sizeof(float) * N3,
                                    dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, r->stream));
    CK(cudaStreamSynchronize(r->stream));
    return check_status(r);
}

int bsg_recon_accumulators(bsg_recon* h, int half, double* vol_out, double* weight_out, int flags) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || half < 0 || half >= r->nhalves) return fail(BSG_ERR_ARG, "bsg_recon_accumulators: bad half %d", half);
    CK(cudaSetDevice(r->device));
    const size_t N3 = r->vol_elems();
    const bool dev = (flags & BSG_DEVICE_PTR) != 0;
    const cudaMemcpyKind k = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    const int zs = r->zsplit, N = r->g.map;
    if (zs > 0 && (!vol_out || !weight_out)) {
        // the map's sums above the split need both channels' mirrors
        if (dev) return fail(BSG_ERR_ARG, "bsg_recon_accumulators: give both outputs with BSG_DEVICE_PTR");
        std::vector<double> tv(vol_out ? 0 : 2 * N3), tw(weight_out ? 0 : N3);
        return bsg_recon_accumulators(h, half, vol_out ? vol_out : tv.data(), weight_out ? weight_out : tw.data(),
                                      flags);
    }
    if (zs > 0 && dev) {
        // half-space form -> the map's sums, on the device
        CK(launch_map_sums(reinterpret_cast<double2*>(vol_out), weight_out, r->d_vol[half], r->d_w[half],
                           r->d_evol[half], r->d_ew[half], N, zs, r->stream));
        CK(cudaStreamSynchronize(r->stream));
        return BSG_OK;
    }
    if (vol_out) CK(cudaMemcpyAsync(vol_out, r->d_vol[half], sizeof(double2) * N3, k, r->stream));
    if (weight_out) CK(cudaMemcpyAsync(weight_out, r->d_w[half], sizeof(double) * N3, k, r->stream));
    std::vector<double> ev, ew;
    if (zs > 0) {
        const size_t n = (size_t)zs * N * N;
        ev.resize(2 * n);
        ew.resize(n);
        CK(cudaMemcpyAsync(ev.data(), r->d_evol[half], sizeof(double2) * n, cudaMemcpyDeviceToHost, r->stream));
        CK(cudaMemcpyAsync(ew.data(), r->d_ew[half], sizeof(double) * n, cudaMemcpyDeviceToHost, r->stream));
    }
    CK(cudaStreamSynchronize(r->stream));
    if (zs > 0) {
        // half-space form -> the map's sums (as launch_map_sums, on the
        // host): above the split from the paired sums below it, then the rest
        const size_t n = N, n2 = n * n;
        for (size_t i = (size_t)zs * n2; i < N3; ++i) {
            const size_t x = i % n, y = (i / n) % n, z = i / n2;
            const size_t m = (((n - z) % n) * n + (n - y) % n) * n + (n - x) % n;
            vol_out[2 * i] += vol_out[2 * m];
            vol_out[2 * i + 1] -= vol_out[2 * m + 1];
            weight_out[i] = weight_out[i] + weight_out[m];
        }
        for (size_t i = 0; i < (size_t)zs * n2; ++i) {
            vol_out[2 * i] += ev[2 * i];
            vol_out[2 * i + 1] += ev[2 * i + 1];
            weight_out[i] += ew[i];
        }
    }
    return BSG_OK;
}

namespace bsg {
// dst[i] += src[i]: one shard's partial sums into the accumulators
__global__ void add_partial_kernel(double* __restrict__ dst, const double* __restrict__ src, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] += src[i];
}
}  // namespace bsg

int bsg_recon_add_partial(bsg_recon* h, int half, const double* vol, const double* weight, const double* power,
                          const double* weight2, int flags) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || half < 0 || half >= r->nhalves) return fail(BSG_ERR_ARG, "bsg_recon_add_partial: bad half %d", half);
    if (!vol || !weight) return fail(BSG_ERR_ARG, "bsg_recon_add_partial: vol and weight are required");
    if ((power == nullptr) != (weight2 == nullptr))
        return fail(BSG_ERR_ARG, "bsg_recon_add_partial: give power and weight2 together");
    if (power && !r->g.fom) return fail(BSG_ERR_STATE, "bsg_recon_add_partial: power sums need fom = 1");
    CK(cudaSetDevice(r->device));
    if (r->zsplit > 0) {
        // the incoming sums are a full map's: this context's become one too
        int rc = set_half_space(r, false);
        if (rc) return rc;
    }
    const size_t N3 = r->vol_elems();
    const bool dev = flags & BSG_DEVICE_PTR;
    double* stage = nullptr;
    if (!dev) {
        // host sums pass through the finishing work buffer (N^3 complex
        // floats = N^3 doubles), in stream order with the gridding
        int rc = ensure_finish_buffers(r);
        if (rc) return rc;
        stage = reinterpret_cast<double*>(r->d_work);
    }
    auto add = [&](double* dst, const double* src, size_t n) -> int {
        for (size_t off = 0; off < n; off += N3) {
            const size_t cnt = std::min(N3, n - off);
            const double* s = src + off;
            if (!dev) {
                CK(cudaMemcpyAsync(stage, s, sizeof(double) * cnt, cudaMemcpyHostToDevice, r->stream));
                s = stage;
            }
            add_partial_kernel<<<148 * 8, 256, 0, r->stream>>>(dst + off, s, cnt);
            CK(cudaGetLastError());
            r->stats.launches += 1;
        }
        return BSG_OK;
    };
    r->dirty = true;            // the accumulators hold sums (a full map's)
    int rc = add(reinterpret_cast<double*>(r->d_vol[half]), vol, 2 * N3);
    if (!rc) rc = add(r->d_w[half], weight, N3);
    if (!rc && power) rc = add(r->d_pow[half], power, N3);
    if (!rc && weight2) rc = add(r->d_w2[half], weight2, N3);
    if (rc) return rc;
    CK(cudaStreamSynchronize(r->stream));
    return BSG_OK;
}

int bsg_recon_fsc(bsg_recon* h, int nshell, double* fsc_out) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || !fsc_out || nshell < 1) return fail(BSG_ERR_ARG, "bsg_recon_fsc: bad argument");
    if (r->nhalves < 2) return fail(BSG_ERR_STATE, "bsg_recon_fsc: needs half maps (nmaps >= 2)");
    CK(cudaSetDevice(r->device));
    const size_t N3 = r->vol_elems();
    for (int i = 0; i < 2; ++i)
        if (!r->d_half_weighed[i]) { int rc = alloc((void**)&r->d_half_weighed[i], sizeof(float2) * N3); if (rc) return rc; }
    if (r->d_fsc) { cudaFree(r->d_fsc); r->d_fsc = nullptr; }
    int rc = alloc((void**)&r->d_fsc, sizeof(double) * 3 * (size_t)r->g.map * nshell + sizeof(double) * nshell);
    if (rc) return rc;
    double* d_out = r->d_fsc + 3 * (size_t)r->g.map * nshell;
    CK(launch_fsc(*r, nshell, d_out, r->stream));
    r->stats.launches += 4;
    CK(cudaMemcpyAsync(fsc_out, d_out, sizeof(double) * nshell, cudaMemcpyDeviceToHost, r->stream));
    CK(cudaStreamSynchronize(r->stream));
    return BSG_OK;
}

int bsg_recon_set_symmetry(bsg_recon* h, const double* ops, int nops) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || nops < 0 || (nops > 0 && !ops)) return fail(BSG_ERR_ARG, "bsg_recon_set_symmetry: bad argument");
    if (nops > 4096) return fail(BSG_ERR_ARG, "bsg_recon_set_symmetry: %d operators (at most 4096)", nops);
    for (int s = 0; s < nops; ++s) {
        // rotations only: rows orthonormal to 1e-6
        const double* S = ops + 9 * s;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                const double d = S[3 * a] * S[3 * b] + S[3 * a + 1] * S[3 * b + 1] + S[3 * a + 2] * S[3 * b + 2];
                if (!(fabs(d - (a == b ? 1.0 : 0.0)) < 1e-6))
                    return fail(BSG_ERR_ARG, "bsg_recon_set_symmetry: operator %d is not a rotation", s);
            }
    }
    r->sym.assign(ops, ops + 9 * (size_t)(nops > 1 ? nops : 0));
    return BSG_OK;
}

int bsg_recon_set_tile_shape(bsg_recon* h, int shape) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r) return fail(BSG_ERR_ARG, "bsg_recon_set_tile_shape: null context");
    CK(cudaSetDevice(r->device));
    return set_shape(r, shape);
}

int bsg_recon_set_half_space(bsg_recon* h, int enable, int* zsplit_out) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r) return fail(BSG_ERR_ARG, "bsg_recon_set_half_space: null context");
    CK(cudaSetDevice(r->device));
    const int rc = set_half_space(r, enable != 0);
    if (rc) return rc;
    if (zsplit_out) *zsplit_out = r->zsplit;
    return BSG_OK;
}

int bsg_recon_autotune(bsg_recon* h, const float* images, const double* params, long nparts, int flags,
                       double* ms_out, int* best_out) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || !images || !params || nparts < 1) return fail(BSG_ERR_ARG, "bsg_recon_autotune: bad argument");
    CK(cudaSetDevice(r->device));
    const bool was_timing = r->timing;
    const bsg_recon_stats saved = r->stats;
    int best = r->shape;
    double best_ms = 1e300;
    for (int sh = 0; sh < insert_num_shapes(); ++sh) {
        if (sh == 3 && r->g.fom) { if (ms_out) ms_out[sh] = -1; continue; }
        int rc = set_shape(r, sh);
        if (rc) return rc;
        rc = bsg_recon_reset(h);
        if (rc) return rc;
        r->timing = true;
        for (auto& t : r->timed) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
        r->timed.clear();
        rc = process(r, images, params, nparts, flags, nullptr);
        if (rc) return rc;
        CK(cudaStreamSynchronize(r->stream));
        double ms = 0;
        for (auto& t : r->timed) {
            float e = 0.f;
            cudaEventElapsedTime(&e, t.a, t.b);
            if (t.kind == 0) ms += e;
            cudaEventDestroy(t.a);
            cudaEventDestroy(t.b);
        }
        r->timed.clear();
        if (ms_out) ms_out[sh] = ms;
        if (ms < best_ms) { best_ms = ms; best = sh; }
    }
    r->timing = was_timing;
    r->stats = saved;
    int rc = set_shape(r, best);
    if (rc) return rc;
    if (best_out) *best_out = best;
    return bsg_recon_reset(h);
}

int bsg_recon_set_timing(bsg_recon* h, int enable) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r) return fail(BSG_ERR_ARG, "bsg_recon_set_timing: null context");
    r->timing = enable != 0;
    return BSG_OK;
}

int bsg_recon_get_stats(bsg_recon* h, bsg_recon_stats* st) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || !st) return fail(BSG_ERR_ARG, "bsg_recon_get_stats: bad argument");
    CK(cudaSetDevice(r->device));
    CK(cudaStreamSynchronize(r->stream));
    CK(cudaStreamSynchronize(r->fft_stream));
    CK(cudaStreamSynchronize(r->copy_stream));
    for (auto& t : r->timed) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t.a, t.b);
        if (t.kind == 0) r->stats.insert_ms += ms;
        else if (t.kind == 1) r->stats.fft2d_ms += ms;
        else r->stats.h2d_ms += ms;
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    r->timed.clear();
    *st = r->stats;
    return check_status(r);
}

int bsg_recon_synchronize(bsg_recon* h) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r) return fail(BSG_ERR_ARG, "bsg_recon_synchronize: null context");
    CK(cudaSetDevice(r->device));
    CK(cudaStreamSynchronize(r->copy_stream));
    CK(cudaStreamSynchronize(r->fft_stream));
    CK(cudaStreamSynchronize(r->stream));
    return check_status(r);
}

void* bsg_recon_stream(bsg_recon* h) {
    Recon* r = reinterpret_cast<Recon*>(h);
    return r ? (void*)r->stream : nullptr;
}

}  // extern "C"

// ---- reconstruction statistics (host, FP64 sums) -----------------------------
namespace {

// Bimage::radial(0, maxrad, 1, wrap = 1) of an N^3 real array about the
// origin 0: value split linearly between the two shells around
// |(x, y, z)|, sums and weights in float as the reference's Float image and
// vector<float> hold them; maxrad is clamped to N / 2.
std::vector<double> radial_average(const std::vector<double>& v, int N, long maxrad) {
    const long h = N / 2;
    if (maxrad < 1 || maxrad > h) maxrad = h;
    std::vector<float> sum(maxrad, 0.f), num(maxrad, 0.f);
    size_t i = 0;
    for (int zz = 0; zz < N; ++zz) {
        double dz = zz > h ? zz - N : zz;
        const double z2 = dz * dz;
        for (int yy = 0; yy < N; ++yy) {
            double dy = yy > h ? yy - N : yy;
            const double y2 = dy * dy;
            for (int xx = 0; xx < N; ++xx, ++i) {
                double dx = xx > h ? xx - N : xx;
                const double r = sqrt(dx * dx + y2 + z2);
                long ir = (long)r;
                if (ir < maxrad) {
                    const double f = r - ir, f1 = 1 - f;
                    num[ir] = (float)((double)num[ir] + f1);
                    sum[ir] = (float)((double)sum[ir] + f1 * v[i]);
                    if (++ir < maxrad) {
                        num[ir] = (float)((double)num[ir] + f);
                        sum[ir] = (float)((double)sum[ir] + f * v[i]);
                    }
                }
            }
        }
    }
    std::vector<double> out(maxrad, 0.0);
    for (long j = 0; j < maxrad; ++j) out[j] = num[j] ? (double)(float)((double)sum[j] / num[j]) : 0.0;
    return out;
}

}  // namespace

int bsg_recon_statistics(bsg_recon* h, int imap, double resolution, bsg_recon_shell_stats* out, double* table,
                         int max_rows) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || !out || imap < 0 || imap > 2 || (imap > 0 && r->nhalves < 2))
        return fail(BSG_ERR_ARG, "bsg_recon_statistics: bad argument (map %d)", imap);
    if (!r->g.fom) return fail(BSG_ERR_STATE, "bsg_recon_statistics: needs the power and weight^2 channels (fom = 1)");
    CK(cudaSetDevice(r->device));
    CK(cudaStreamSynchronize(r->stream));
    const int N = r->g.map;
    const size_t N3 = r->vol_elems();
    // the map's sums: one half, or both added (imap 0 with half maps)
    std::vector<double> v(2 * N3), w(N3), p(N3), q(N3);
    const int h0 = (r->nhalves == 2 && imap > 0) ? imap - 1 : 0;
    CK(cudaMemcpy(v.data(), r->d_vol[h0], sizeof(double2) * N3, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(w.data(), r->d_w[h0], sizeof(double) * N3, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(p.data(), r->d_pow[h0], sizeof(double) * N3, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(q.data(), r->d_w2[h0], sizeof(double) * N3, cudaMemcpyDeviceToHost));
    if (r->nhalves == 2 && imap == 0) {
        std::vector<double> t(2 * N3);
        CK(cudaMemcpy(t.data(), r->d_vol[1], sizeof(double2) * N3, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < 2 * N3; ++i) v[i] += t[i];
        t.resize(N3);
        CK(cudaMemcpy(t.data(), r->d_w[1], sizeof(double) * N3, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < N3; ++i) w[i] += t[i];
        CK(cudaMemcpy(t.data(), r->d_pow[1], sizeof(double) * N3, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < N3; ++i) p[i] += t[i];
        CK(cudaMemcpy(t.data(), r->d_w2[1], sizeof(double) * N3, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < N3; ++i) q[i] += t[i];
    }
    // fspace_reconstruction_weigh (Bimage_reconstruct.cpp:486-515); the map
    // held as float complex as the reference holds it
    std::vector<float> fr(N3), fi(N3);
    long cov = 0;
    for (size_t i = 0; i < N3; ++i) {
        if (w[i] > 1e-30) {
            q[i] = w[i] - q[i] / w[i];
            fr[i] = (float)(v[2 * i] / w[i]);
            fi[i] = (float)(v[2 * i + 1] / w[i]);
            if (q[i] > 1) p[i] /= q[i];
            else if (w[i] > 1) p[i] /= w[i];
            if (p[i] < 0) p[i] = 0;
            ++cov;
        } else {
            fr[i] = fi[i] = 0.f;
            p[i] = 0;
            w[i] = q[i] = 1e-30;
        }
    }
    p[0] = 1;
    const double real = r->g.mscale, samp = r->cfg.map_sampling;
    // coverage against the sphere of fspace_maximum_radius(hi_res) + 1
    auto max_radius = [&](double res) -> long { return res > 0.1 ? (long)(real / res) : (long)(N / 2.0); };
    const double rad = (double)max_radius(resolution) + 1;
    out->coverage = cov;
    out->coverage_pct = cov * 100.0 / ((4.0 / 3.0) * M_PI * rad * rad * rad);
    // Bimage::friedel_check (Bimage_fspace.cpp:2024-2066)
    {
        double s = 0, Rr = 0, Ri = 0;
        for (int zz = 0; zz < N; ++zz) {
            const int zf = zz ? N - zz : 0;
            for (int yy = 0; yy < N; ++yy) {
                const int yf = yy ? N - yy : 0;
                for (int xx = 0; xx < (N + 1) / 2; ++xx) {
                    const int xf = xx ? N - xx : 0;
                    const size_t i = ((size_t)zz * N + yy) * N + xx, j = ((size_t)zf * N + yf) * N + xf;
                    const double vr = fr[i], vi = fi[i], ur = fr[j], ui = fi[j];
                    const double ww = ((vr * vr + vi * vi) + (ur * ur + ui * ui)) / 2;
                    double d = vr - ur;
                    Rr += d * d * ww;
                    d = vi + ui;
                    Ri += d * d * ww;
                    s += ww;
                }
            }
        }
        Rr = sqrt(Rr / s);
        Ri = sqrt(Ri / s);
        out->friedel = sqrt(Rr * Rr + Ri * Ri);
    }
    // fspace_reconstruction_stats (Bimage_reconstruct.cpp:526-599)
    const long maxrad = max_radius(resolution);
    double res_checked = resolution;         // fspace_radial_power's check_resolution
    if (res_checked > real) res_checked = real;
    else res_checked = std::max(res_checked, 2.0 / sqrt(3.0 / (samp * samp)));
    const long maxrad_p = max_radius(res_checked);
    std::vector<double> prad(std::max(0L, maxrad_p), 0.0);
    {
        std::vector<float> sum(prad.size(), 0.f), num(prad.size(), 0.f);
        const long hh = (N - 1) / 2;
        const double fsc_ = 1.0 / real;
        size_t i = 0;
        for (int zz = 0; zz < N; ++zz) {
            double rz = zz > hh ? zz - N : zz;
            rz *= fsc_;
            rz *= rz;
            for (int yy = 0; yy < N; ++yy) {
                double ry = yy > hh ? yy - N : yy;
                ry *= fsc_;
                ry *= ry;
                for (int xx = 0; xx < N; ++xx, ++i) {
                    double rx = xx > hh ? xx - N : xx;
                    rx *= fsc_;
                    rx *= rx;
                    const double radius = real * sqrt(rx + ry + rz);
                    long ir = (long)radius;
                    if (ir < maxrad_p) {
                        const double f = radius - ir, f1 = 1 - f;
                        const double val = (double)fr[i] * fr[i] + (double)fi[i] * fi[i];
                        num[ir] = (float)((double)num[ir] + f1);
                        sum[ir] = (float)((double)sum[ir] + f1 * val);
                        if (++ir < maxrad_p) {
                            num[ir] = (float)((double)num[ir] + f);
                            sum[ir] = (float)((double)sum[ir] + f * val);
                        }
                    }
                }
            }
        }
        for (size_t j = 0; j < prad.size(); ++j) prad[j] = num[j] ? (double)(float)((double)sum[j] / num[j]) : 0.0;
    }
    const std::vector<double> pfom = radial_average(p, N, maxrad), pw = radial_average(w, N, maxrad),
                              pw2 = radial_average(q, N, maxrad);
    auto at = [](const std::vector<double>& a, long k) { return k >= 0 && k < (long)a.size() ? a[k] : 0.0; };
    double fscp = 1, snrp = 10, res_fsc = 0, res_snr = 0;
    const double fsc_cut = 0.3, snr_cut = 0.5;
    int rows = 0;
    for (long i = 1; i < maxrad; ++i, ++rows) {
        const double s = i / real, res = real / i;
        double fsc = 0, snr = 0, signal = 0, noise = 0;
        const double wi = at(pw, i);
        if (wi > 1e-3) {
            const double w2 = at(pw2, i);
            noise = (at(pfom, i) - at(prad, i)) / w2;
            signal = (wi * at(prad, i) - at(pfom, i)) / w2;
            if (noise > 0) snr = signal / noise;
            fsc = snr / (snr + 1);
            if (fsc < 0) fsc = 0;
        }
        if (fscp >= fsc_cut && fsc < fsc_cut) res_fsc = 1 / (s - (fsc_cut - fsc) / ((fscp - fsc) * real));
        if (snrp >= snr_cut && snr < snr_cut) res_snr = 1 / (s - (snr_cut - snr) / ((snrp - snr) * real));
        fscp = fsc;
        snrp = snr;
        if (table && rows < max_rows) {
            double* t = table + (size_t)rows * BSG_STATS_COLUMNS;
            t[0] = (double)i; t[1] = s; t[2] = res; t[3] = wi; t[4] = at(prad, i);
            t[5] = signal; t[6] = noise; t[7] = snr; t[8] = fsc;
        }
    }
    out->rows = rows;
    out->res_snr = res_snr;
    out->res_fsc = res_fsc;
    return BSG_OK;
}

int bsg_recon_set_symmetrize(bsg_recon* h, const double* axes, const int* orders, int nops) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || nops < 0 || nops > 8 || (nops > 0 && (!axes || !orders)))
        return fail(BSG_ERR_ARG, "bsg_recon_set_symmetrize: bad argument (nops %d)", nops);
    for (int i = 0; i < nops; ++i)
        if (orders[i] < 1 || orders[i] > 9)
            return fail(BSG_ERR_ARG, "bsg_recon_set_symmetrize: operation %d has order %d (1..9)", i, orders[i]);
    r->symz_axes.assign(axes, axes + 3 * nops);
    r->symz_orders.assign(orders, orders + nops);
    return BSG_OK;
}

int bsg_recon_set_rescale(bsg_recon* h, double avg, double std) {
    Recon* r = reinterpret_cast<Recon*>(h);
    if (!r || !std::isfinite(avg) || !std::isfinite(std)) return fail(BSG_ERR_ARG, "bsg_recon_set_rescale: bad argument");
    r->rescale_avg = avg;
    r->rescale_std = std > 0 ? std : 0;
    return BSG_OK;
}
