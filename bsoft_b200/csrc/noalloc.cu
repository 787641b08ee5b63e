// noalloc.cu - bsg_particle_spectra_noalloc: the 2-D particle stage (pad,
// FFT, origin shift, CTF) for callers that must not have the library
// allocate device memory.
//
// Who needs it: programs that own all of the GPU's memory through their own
// pool or arena (a streaming pipeline that reserves its memory at start-up
// so that a long run never stalls in, or fragments memory through,
// cudaMalloc; a host application that forbids device allocations after its
// initialisation).  Such callers pass their own device buffers for the
// particle images and the spectra; everything else the kernels need lives
// in one fixed scratch area that is part of the loaded library.
//
// The scratch area is a file-scope __device__ array of SCRATCH_BYTES
// (64 MiB).  Every GPU that loads the library holds it until the process
// exits.  Host code cannot use the array's name as a device address, so the
// first call on each device looks its address up with
// cudaGetSymbolAddress, with that device current, and keeps it; make that
// first call before any stream capture.  All calls share the one array:
// calls whose work overlaps on the GPU (different streams, or different
// host threads on one device) race on it and must be serialised by the
// caller.  Nothing in the array has to start at zero: every word the
// kernels read is written earlier in the same call.
#include "context.cuh"
#include "fft_dev.cuh"

#include <math.h>
#include <mutex>

namespace bsg {

constexpr size_t SCRATCH_BYTES = BSG_NOALLOC_SCRATCH_BYTES;

static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

cudaError_t launch_background(const Context& c, const float* img, int nimg, cudaStream_t s);
cudaError_t launch_rows(const Context& c, const float* img, int nimg, cudaStream_t s);
cudaError_t launch_cols(const Context& c, int nimg, float2* spectra, cudaStream_t s);
cudaError_t prepare_fft2d_attributes();
void set_error(const char* fmt, ...);

namespace {

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void* g_addr[MAX_DEVICES] = {};
// host staging of the particle records: more than the scratch area can hold
// at the smallest transform (32^2: about 10 KB of scratch per particle)
constexpr long MAX_RECORDS = 8192;
DevParticle g_records[MAX_RECORDS];

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Scratch layout for `np` particles of box n and transform edge ft.
struct Layout {
    size_t tw, part, bkg, phase, rows, spec, total;
};

Layout layout(int n, int ft, long np) {
    Layout L;
    size_t off = 0;
    L.tw = off;    off += align256(sizeof(float2) * (size_t)(ft / 2));
    L.part = off;  off += align256(sizeof(DevParticle) * (size_t)np);
    L.bkg = off;   off += align256(sizeof(double) * (size_t)np);
    L.phase = off; off += align256(sizeof(float2) * 2 * (size_t)ft * np);
    L.rows = off;  off += align256(sizeof(float2) * (size_t)n * (ft / 2 + 1) * np);
    L.spec = off;  off += align256(sizeof(float2) * (size_t)(ft + 1) * (ft + 2) * np);
    L.total = off;
    return L;
}

__global__ void twiddle_kernel(float2* tw, int ft) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < ft / 2; j += gridDim.x * blockDim.x) {
        double s, c;
        sincos(-2.0 * 3.14159265358979323846 * j / ft, &s, &c);
        tw[j] = make_float2((float)c, (float)s);
    }
}

// centred [k + ft/2][h + ft/2] (pitch ft + 2) -> reference pixel order
__global__ void to_reference_order(const float2* spec, int ft, long np, float2* out) {
    const int hf = ft / 2, pitch = ft + 2;
    const size_t per = (size_t)ft * ft;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < per * np; i += (size_t)gridDim.x * blockDim.x) {
        const size_t p = i / per;
        const int yy = (int)((i % per) / ft), xx = (int)(i % ft);
        const int k = sfreq(yy, ft), h = sfreq(xx, ft);
        out[i] = spec[p * (size_t)(ft + 1) * pitch + (size_t)(k + hf) * pitch + (h + hf)];
    }
}

// Host copy of the 32-double particle record into the device layout (the
// same arithmetic as the context path in capi.cu).
void to_dev_particle(const Geometry& g, const double* q, DevParticle& d) {
    memset(&d, 0, sizeof(d));
    d.shx = q[0] / g.ft * 2.0 * M_PI;
    d.shy = q[1] / g.ft * 2.0 * M_PI;
    d.bx = q[2];
    d.by = q[3];
    const double pixel = q[13];
    d.fs = 1.0 / (g.ft * pixel);
    d.c00 = q[16]; d.c20 = q[17]; d.c22 = q[18]; d.c2m2 = q[19]; d.c40 = q[20]; d.c11 = q[21]; d.c1m1 = q[22];
    d.half = (int)q[23];
    d.na = q[24] != 0 ? q[24] : 1.0;
    d.nb = q[24] != 0 ? q[25] : 0.0;
}

}  // namespace

}  // namespace bsg

using namespace bsg;

extern "C" int bsg_particle_spectra_noalloc(const bsg_recon_config* cfg, const float* d_images, const double* params,
                                            long nparts, float* d_out, void* stream) {
    if (!cfg || !d_images || !params || !d_out || nparts < 1) {
        set_error("bsg_particle_spectra_noalloc: null pointer or no particles");
        return BSG_ERR_ARG;
    }
    const int n = cfg->n, ft = cfg->ft;
    if (n < 2 || ft < 32 || ft > 1024 || (ft & (ft - 1)) || ft < n) {
        set_error("bsg_particle_spectra_noalloc: transform size %d must be a power of two in [32, 1024] and >= box %d",
                  ft, n);
        return BSG_ERR_ARG;
    }
    if (cfg->interp < 0 || cfg->interp > 2 || cfg->ctf_action < 0 || !(cfg->hi_res > 0)) {
        set_error("bsg_particle_spectra_noalloc: interp %d, ctf_action %d or resolution %g out of range",
                  cfg->interp, cfg->ctf_action, cfg->hi_res);
        return BSG_ERR_ARG;
    }
    // bound the particle count before multiplying it into the layout
    const size_t one = layout(n, ft, 1).total;
    const long fit = (long)(SCRATCH_BYTES / one);
    const long cap = fit < MAX_RECORDS ? fit : MAX_RECORDS;
    if (nparts > cap || layout(n, ft, nparts).total > SCRATCH_BYTES) {
        set_error("bsg_particle_spectra_noalloc: %ld particles of box %d (transform %d) do not fit the fixed "
                  "scratch area of %zu bytes (at most %ld particles of this size per call)",
                  nparts, n, ft, SCRATCH_BYTES, cap);
        return BSG_ERR_ARG;
    }
    const Layout L = layout(n, ft, nparts);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
        set_error("bsg_particle_spectra_noalloc: no current CUDA device (%s)", cudaGetErrorString(e));
        return BSG_ERR_NODEV;
    }
    void* base;
    {
        // once per device, with that device current: the scratch array's
        // device address (and the kernels' shared-memory limits)
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                set_error("bsg_particle_spectra_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
                return BSG_ERR_CUDA;
            }
            e = prepare_fft2d_attributes();
            if (e != cudaSuccess) {
                set_error("bsg_particle_spectra_noalloc: kernel set-up failed: %s", cudaGetErrorString(e));
                return BSG_ERR_CUDA;
            }
            g_addr[dev] = p;
        }
        base = g_addr[dev];
    }
    unsigned char* sc = static_cast<unsigned char*>(base);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // a context on the stack whose buffers all point into the scratch area
    Context c;
    c.cfg = *cfg;
    c.g.n = n;
    c.g.ft = ft;
    c.g.map = cfg->map;
    c.g.logft = ilog2i(ft);
    c.g.interp = cfg->interp;
    c.g.ctf_action = cfg->ctf_action;
    c.g.wiener = cfg->wiener;
    c.g.ctf_shi2 = 1.0 / (cfg->hi_res * cfg->hi_res);
    c.d_tw = reinterpret_cast<float2*>(sc + L.tw);
    c.d_part = reinterpret_cast<DevParticle*>(sc + L.part);
    c.d_bkg = reinterpret_cast<double*>(sc + L.bkg);
    c.d_phase = reinterpret_cast<float2*>(sc + L.phase);
    c.d_rows = reinterpret_cast<float2*>(sc + L.rows);
    float2* spec = reinterpret_cast<float2*>(sc + L.spec);

    // particle records: converted on the host into one static buffer and
    // sent in one copy.  The buffer is ordinary (pageable) host memory, so
    // CUDA stages the copy before cudaMemcpyAsync returns, after which the
    // buffer may be refilled; the lock keeps two host threads from filling
    // it at once.
    for (long i = 0; i < nparts; ++i) {
        const double* q = params + i * BSG_PARTICLE_DOUBLES;
        if (!(q[13] > 0)) {
            set_error("bsg_particle_spectra_noalloc: particle %ld has pixel size %g", i, q[13]);
            return BSG_ERR_ARG;
        }
    }
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (long i = 0; i < nparts; ++i) to_dev_particle(c.g, params + i * BSG_PARTICLE_DOUBLES, g_records[i]);
        e = cudaMemcpyAsync(c.d_part, g_records, sizeof(DevParticle) * nparts, cudaMemcpyHostToDevice, s);
    }
    if (e != cudaSuccess) {
        set_error("bsg_particle_spectra_noalloc: copying particle records: %s", cudaGetErrorString(e));
        return BSG_ERR_CUDA;
    }
    twiddle_kernel<<<1, 256, 0, s>>>(c.d_tw, ft);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = launch_background(c, d_images, (int)nparts, s);
    if (e == cudaSuccess) e = launch_rows(c, d_images, (int)nparts, s);
    if (e == cudaSuccess) e = launch_cols(c, (int)nparts, spec, s);
    if (e == cudaSuccess) {
        to_reference_order<<<148 * 4, 256, 0, s>>>(spec, ft, nparts, reinterpret_cast<float2*>(d_out));
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_error("bsg_particle_spectra_noalloc: launch failed: %s", cudaGetErrorString(e));
        return BSG_ERR_CUDA;
    }
    return BSG_OK;
}
