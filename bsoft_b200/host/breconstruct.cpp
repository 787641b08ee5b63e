// breconstruct - drop-in for the reference's breconstruct (bsoft/src/
// breconstruct.cpp) on one B200: reads the same STAR project and MRC particle
// stacks, plans the reconstruction by the reference's rules and drives
// libbsgpu's C ABI (include/bsgpu.h) for the per-particle work, the weighing,
// the inverse transform and the sinc correction.
//
// Options (the reference's spelling, breconstruct.cpp:25-67):
//   -interpolation nearest|weighted|trilinear   (default nearest)
//   -pad 2          -CTF none|flip|apply|correct|wiener    -wiener 0.2
//   -resolution 4   -size 64   -sampling 1.5   -scale 1
//   -fullmap / -halfmaps       -bootstrap     -symmetry D6 (inserted during reconstruction)
//   -reconstruction out.mrc    -fom fom.mrc    -batch 4096   -device 0
//   -plan           print the per-particle records (no GPU work) and exit
// Output names follow the reference: out.mrc for a full map, out_01.mrc and
// out_02.mrc for half maps (breconstruct.cpp:362-377).
//
// Project reading follows read_project / rwmgSTAR.cpp (particle loop
// :195-262, CTF block :458-519, micrograph block :521-655) and rwmg.cpp:
// 650-659; planning follows breconstruct.cpp:190-245, project_set_
// reconstruction_size (mg_reconstruct.cpp:596-651), part_ft_size (:38-64),
// Bimage::check_resolution (Bimage.cpp:633-648) and the per-particle set-up
// of particle_reconstruct (mg_reconstruct.cpp:143-212).
#include "bsgpu.h"
#include "project.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include <unistd.h>

namespace {

using namespace bsh;

// ---------------------------------------------------------------- plan
struct Options {
    int interp = 0, pad = 2, ctf_action = 0, size = 0, nmaps = 0, batch = 4096, device = 0;
    double wiener = 0, resolution = 0, sampling = 0, scale = 1;
    bool bootstrap = false, plan_only = false;
    int verbose = 0;
    int sym_mode = 0;               // -mode: 0 during reconstruction, 1 after it, 2 random view
    int threads = 2;                // -threads: the reference's partial maps (-mode 2's draw order)
    long seed = -1;                 // -seed: random() seed of -mode 2 (default: the process id)
    double rescale_avg = 0, rescale_std = 0;   // -rescale avg,std (std > 0: on)
    bool ewald = false;             // -ewald: Ewald-sphere insertion
    std::string symmetry = "C1";
    std::string recons, fom;
    std::vector<std::string> inputs;
};

long next_pow2(long n) { long p = 1; while (p < n) p *= 2; return p; }

// mg_reconstruct.cpp:38-64
long part_ft_size(long xsize, double scale, int pad) {
    long ft = xsize;
    if (scale > 1) ft = (long)(xsize * scale);
    if (pad < 1) return ft;
    pad = std::min(pad, 8);
    ft = next_pow2((long)(pad * xsize * scale));
    if (ft < xsize) ft = next_pow2(xsize);
    return ft;
}

struct Plan {
    int n = 0, ft = 0, map = 0, nmaps = 1;
    double map_sampling = 0, hi_res = 0, wiener = 0;
    double resolution = 0;          // the limit before check_resolution (the statistics use it)
    std::vector<double> rec;                        // BSG_PARTICLE_DOUBLES per particle
    std::vector<std::pair<int, long>> src;          // (micrograph, image index) per particle
};

// breconstruct -mode 2: every particle inserted once, with a random one of its
// symmetry-related views (random_symmetric_view, bsoft/src/util/
// symmetry.cpp:816-832, called per particle by particle_reconstruct,
// mg_reconstruct.cpp:175).  random() is seeded once (srandom(getpid()),
// random_numbers.cpp:41-48; -seed replaces the process id); per particle the
// index is floor(order random() 0.99999 / get_rand_max()) in long double, and
// get_rand_max() draws 100 numbers of its own after the index's draw
// (random_numbers.cpp:22-30).  Particles draw partial map by partial map (k
// mod T, T = the reference's thread_limit, breconstruct.cpp:204-205), the
// order of its OpenMP loop on one thread.
void random_symmetric_views(Plan& p, const Options& o) {
    const std::vector<double> S = symmetry_operators(o.symmetry);
    const long order = (long)(S.size() / 9), np = (long)p.src.size();
    if (order < 2 || np < 1) return;
    long t = std::max(2, o.threads);
    t = std::max(1L, std::min(t, np / 2));
    if ((p.nmaps & 2) && (t % 2)) ++t;
    srandom((unsigned)(o.seed >= 0 ? o.seed : (long)getpid()));
    for (long m = 0; m < t; ++m)
        for (long k = m; k < np; k += t) {
            const long r = random();
            long rand_max = 32767;
            for (int j = 0; j < 100; ++j)
                if (random() > rand_max) rand_max = 2147483647;
            const long i = (long)((long double)(order * r) * 0.99999L / (long double)rand_max);
            double* R = &p.rec[k * BSG_PARTICLE_DOUBLES + 4];
            const double* G = &S[9 * i];
            double out[9];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    out[3 * a + b] = G[3 * a] * R[b] + G[3 * a + 1] * R[3 + b] + G[3 * a + 2] * R[6 + b];
            std::copy(out, out + 9, R);
        }
}

Plan plan_reconstruction(const std::vector<Micrograph>& mgs, const Options& o) {
    int first = -1;
    for (size_t i = 0; i < mgs.size(); ++i)
        if (!mgs[i].part_id.empty()) { first = (int)i; break; }
    if (first < 0) throw std::runtime_error("no particles");
    const Micrograph& m0 = mgs[first];
    const StackHeader h0 = read_stack_header(m0.particle_file);
    // project_set_reconstruction_size (mg_reconstruct.cpp:596-651)
    double sam = o.sampling;
    if (sam < 0.1) sam = m0.pixel[0] > 0 ? m0.pixel[0] : 0.0;
    if (sam < 0.1) sam = m0.pixel_size;
    if (sam < 0.1) sam = h0.sampling(0);
    Plan p;
    p.n = h0.nx();
    p.map = o.size ? o.size : (int)(h0.nx() * o.scale);
    const double resolution = o.resolution >= 0.1 ? o.resolution : sam;
    long ft = m0.box ? m0.box : h0.nx();
    if (p.map > ft) ft = p.map;
    p.ft = (int)part_ft_size(ft, 1, o.pad);
    p.map_sampling = sam / o.scale;
    // Bimage::check_resolution (Bimage.cpp:633-648) for the cubic map
    double hr = resolution;
    if (hr > p.map * p.map_sampling) hr = p.map * p.map_sampling;
    else hr = std::fmax(hr, 2.0 / std::sqrt(3.0 / (p.map_sampling * p.map_sampling)));
    p.hi_res = hr;
    p.resolution = resolution;
    p.wiener = (o.ctf_action > 2 && o.wiener < 0.01) ? 0.2 : o.wiener;
    p.nmaps = o.nmaps < 1 ? 1 : (o.nmaps > 3 ? 3 : o.nmaps);
    // per-particle records (particle_reconstruct, mg_reconstruct.cpp:143-212)
    long k = 0;
    Ctf em;     // CTFparam defaults for micrographs without a CTF block
    for (size_t mi = 0; mi < mgs.size(); ++mi) {
        const Micrograph& mg = mgs[mi];
        if (mg.part_id.empty()) continue;
        const StackHeader h = read_stack_header(mg.particle_file);
        if (mg.has_ctf) em = mg.ctf;
        for (size_t i = 0; i < mg.part_id.size(); ++i) {
            if (mg.select[i] <= 0) continue;
            const double fo[2] = {h.image_origin(0, mg.part_id[i] - 1), h.image_origin(1, mg.part_id[i] - 1)};
            double r[BSG_PARTICLE_DOUBLES] = {};
            double ox = mg.ox[i], oy = mg.oy[i];
            if (ox <= 0) { ox = fo[0] > 0 ? fo[0] : 0; oy = fo[0] > 0 ? fo[1] : 0; }
            r[0] = ox; r[1] = oy;
            r[2] = fo[0]; r[3] = fo[1];
            view_matrix(mg.vx[i], mg.vy[i], mg.vz[i], mg.va[i], r + 4);
            r[13] = mg.pixel[i] > 0 ? mg.pixel[i] : h.sampling(0);
            r[14] = mg.mag[i] > 0 ? 1.0 / mg.mag[i] : 1.0;
            r[15] = o.bootstrap ? (double)mg.select[i] : 1.0;
            Ctf c = em;
            if (mg.defocus[i] > 0) c.defocus = mg.defocus[i];
            c.coefficients(r + 16);
            // round-robin partial maps; even maps form half 1 (mg_reconstruct.cpp:757-763, 283-290)
            r[23] = (double)(k % 2);
            // particle_reconstruct: ew_wl = em_ctf.lambda() (mg_reconstruct.cpp:209-210)
            if (o.ewald) r[26] = c.lambda();
            if (o.rescale_std > 0) {
                // particle_reconstruct: rescale_to_avg_std(0, 1) with the
                // statistics read_img attaches (mg_reconstruct.cpp:155)
                double avg = h.mean(), sd = h.stddev();
                if (sd < 1e-30) {
                    std::vector<float> img((size_t)h.nx() * h.ny());
                    read_stack_images(mg.particle_file, h, mg.part_id[i] - 1, 1, img.data());
                    double s1 = 0, s2 = 0;
                    for (float v : img) { s1 += v; s2 += (double)v * v; }
                    avg = s1 / img.size();
                    sd = s2 / img.size() - avg * avg;
                    sd = sd > 0 ? std::sqrt(sd) : 0.0;
                }
                const double scale = sd > 1e-30 ? 1.0 / sd : 1.0;
                r[24] = scale;
                r[25] = 0.0 - avg * scale;
            }
            p.rec.insert(p.rec.end(), r, r + BSG_PARTICLE_DOUBLES);
            p.src.push_back({(int)mi, mg.part_id[i] - 1});
            ++k;
        }
    }
    if (o.sym_mode == 2) random_symmetric_views(p, o);
    return p;
}

void usage() {
    fprintf(stderr,
            "Usage: breconstruct [options] input.star\n"
            "  -interpolation nearest|weighted|trilinear  -pad 2  -CTF none|flip|apply|correct|wiener\n"
            "  -wiener 0.2  -resolution 4  -size 64  -sampling 1.5  -scale 1  -fullmap  -halfmaps\n"
            "  -bootstrap  -ewald  -rescale avg,std  -mode 0|1|2  -seed 1  -threads 2  -reconstruction out.mrc\n"
            "  -fom fom.mrc  -verbose 1\n"
            "  -batch 4096  -device 0  -plan\n");
}

int ctf_code(const std::string& v) {
    // Boption::ctf_action (options.h:418-442): flip, apply, correct, wiener
    if (v.empty() || v == "none") return 0;
    if (v[0] == 'f') return 1;
    if (v[0] == 'a') return 2;
    if (v[0] == 'c') return 3;
    if (v[0] == 'w') return 4;
    return atoi(v.c_str());
}

Options parse(int argc, char** argv) {
    Options o;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto val = [&]() -> std::string {
            if (i + 1 >= argc) throw std::runtime_error("option " + a + " needs a value");
            return argv[++i];
        };
        if (a.size() > 1 && a[0] == '-' && a[1] == '-') a = a.substr(1);
        if (a == "-interpolation" || a == "-interp") {
            const std::string v = val();
            o.interp = v[0] == 't' ? 2 : (v[0] == 'w' ? 1 : 0);
        } else if (a == "-pad") o.pad = atoi(val().c_str());
        else if (a == "-CTF") o.ctf_action = ctf_code(val());
        else if (a == "-wiener") { o.wiener = atof(val().c_str()); if (o.wiener < 0.01) o.wiener = 0.01; }
        else if (a == "-resolution") o.resolution = atof(val().c_str());
        else if (a == "-size") o.size = atoi(val().c_str());
        else if (a == "-sampling") o.sampling = atof(val().c_str());
        else if (a == "-scale") o.scale = atof(val().c_str());
        else if (a == "-fullmap") o.nmaps += 1;
        else if (a == "-halfmaps") o.nmaps += 2;
        else if (a == "-bootstrap") o.bootstrap = true;
        else if (a == "-symmetry" || a == "-sym") o.symmetry = val();
        else if (a == "-reconstruction") o.recons = val();
        else if (a == "-fom") o.fom = val();
        else if (a == "-batch") o.batch = atoi(val().c_str());
        else if (a == "-device") o.device = atoi(val().c_str());
        else if (a == "-plan") o.plan_only = true;
        else if (a == "-verbose") o.verbose = atoi(val().c_str());
        else if (a == "-ewald") o.ewald = true;
        else if (a == "-rescale") {
            const std::string v = val();
            const size_t cpos = v.find(',');
            if (cpos == std::string::npos) throw std::runtime_error("-rescale: both average and standard deviation must be given");
            o.rescale_avg = atof(v.c_str());
            o.rescale_std = atof(v.c_str() + cpos + 1);
            if (!(o.rescale_std > 0)) throw std::runtime_error("-rescale: a positive standard deviation must be given");
        }
        else if (a == "-mode") {
            o.sym_mode = atoi(val().c_str());
            if (o.sym_mode < 0 || o.sym_mode > 2)
                throw std::runtime_error("-mode " + std::to_string(o.sym_mode) +
                                         ": 0 (during), 1 (after reconstruction) or 2 (random view)");
        }
        else if (a == "-threads") o.threads = atoi(val().c_str());
        else if (a == "-seed") o.seed = atol(val().c_str());
        else if (a == "-h" || a == "-help") { usage(); exit(0); }
        else if (a[0] == '-') throw std::runtime_error("unknown option " + a);
        else o.inputs.push_back(a);
    }
    if (o.inputs.empty()) throw std::runtime_error("no parameter file given");
    return o;
}

// out.mrc -> out_01.mrc (breconstruct.cpp:362-377)
std::string map_name(const std::string& base, int imap) {
    if (!imap) return base;
    const size_t dot = base.find_last_of('.');
    char tag[16];
    snprintf(tag, sizeof(tag), "_%02d", imap);
    if (dot == std::string::npos) return base + tag;
    return base.substr(0, dot) + tag + base.substr(dot);
}

#define CALL(x)                                                                 \
    do {                                                                        \
        if ((x) != BSG_OK) throw std::runtime_error(std::string(#x) + ": " + bsg_last_error()); \
    } while (0)

}  // namespace

int main(int argc, char** argv) {
    try {
        const Options o = parse(argc, argv);
        std::vector<Micrograph> mgs;
        for (auto& f : o.inputs) {
            auto m = read_project(f);
            mgs.insert(mgs.end(), m.begin(), m.end());
        }
        const Plan p = plan_reconstruction(mgs, o);
        const long np = (long)p.src.size();
        const std::vector<double> sym = symmetry_operators(o.symmetry);
        if (o.plan_only) {
            printf("n %d ft %d map %d map_sampling %.17g hi_res %.17g wiener %.17g nmaps %d particles %ld nsym %ld\n",
                   p.n, p.ft, p.map, p.map_sampling, p.hi_res, p.wiener, p.nmaps, np, (long)(sym.size() / 9));
            for (long i = 0; i < np; ++i) {
                for (int j = 0; j < BSG_PARTICLE_DOUBLES; ++j)
                    printf("%.17g%c", p.rec[i * BSG_PARTICLE_DOUBLES + j], j + 1 < BSG_PARTICLE_DOUBLES ? ' ' : '\n');
            }
            return 0;
        }
        if (o.recons.empty()) throw std::runtime_error("no -reconstruction file name given");
        bsg_recon_config cfg = {};
        cfg.n = p.n; cfg.ft = p.ft; cfg.map = p.map; cfg.map_sampling = p.map_sampling; cfg.hi_res = p.hi_res;
        cfg.interp = o.interp; cfg.ctf_action = o.ctf_action; cfg.wiener = p.wiener; cfg.nmaps = p.nmaps;
        // the power and weight^2 channels: for the -fom map, and for the
        // statistics -verbose prints
        cfg.fom = (o.fom.empty() && !o.verbose) ? 0 : 1; cfg.batch = 0; cfg.device = o.device;
        bsg_recon* rec = nullptr;
        CALL(bsg_recon_create(&cfg, &rec));
        if (o.rescale_std > 0) CALL(bsg_recon_set_rescale(rec, o.rescale_avg, o.rescale_std));
        if (o.sym_mode == 1) {
            // symmetry after reconstruction (mode 1): insert once, symmetrize
            // the finished map (Bimage::symmetrize, breconstruct.cpp:335)
            std::vector<double> ax;
            std::vector<int> ord;
            for (const SymOp& g : symmetry_generators(o.symmetry)) {
                ax.insert(ax.end(), g.a, g.a + 3);
                ord.push_back(g.order);
            }
            CALL(bsg_recon_set_symmetrize(rec, ax.data(), ord.data(), (int)ord.size()));
        } else if (o.sym_mode == 0) {
            // point-group symmetry during reconstruction (mode 0)
            CALL(bsg_recon_set_symmetry(rec, sym.data(), (int)(sym.size() / 9)));
        }   // mode 2: the records already carry each particle's random view
        // stream the particles in host batches (the library uploads and
        // overlaps them with the device work)
        const long n2 = (long)p.n * p.n;
        const long B = std::max(1, o.batch);
        std::vector<float> buf[2] = {std::vector<float>(B * n2), std::vector<float>(B * n2)};
        std::map<int, StackHeader> hdrs;
        for (long b0 = 0, bi = 0; b0 < np; b0 += B, ++bi) {
            const long cnt = std::min(B, np - b0);
            std::vector<float>& dst = buf[bi % 2];
            if (bi >= 2) CALL(bsg_recon_synchronize(rec));   // the buffer's previous upload has finished
            for (long i = 0; i < cnt; ++i) {
                const auto& s = p.src[b0 + i];
                const Micrograph& mg = mgs[s.first];
                if (!hdrs.count(s.first)) hdrs[s.first] = read_stack_header(mg.particle_file);
                read_stack_images(mg.particle_file, hdrs[s.first], s.second, 1, dst.data() + i * n2);
            }
            CALL(bsg_recon_insert(rec, dst.data(), p.rec.data() + b0 * BSG_PARTICLE_DOUBLES, cnt, 0));
        }
        CALL(bsg_recon_synchronize(rec));
        const size_t n3 = (size_t)p.map * p.map * p.map;
        std::vector<float> vol(n3), fom(cfg.fom ? n3 : 0);
        const int flags = o.interp == 2 ? BSG_SINC : 0;
        if (o.verbose) {
            // img_reconstruction_sum_weigh's report (mg_reconstruct.cpp:328-349):
            // Friedel residual and coverage of every map, the shell table of
            // the first (Bimage_reconstruct.cpp:526-599), in its format
            for (int i = 0; i < p.nmaps; ++i) {
                const int imap = p.nmaps == 2 ? i + 1 : (p.nmaps == 3 ? i : 0);
                bsg_recon_shell_stats st;
                std::vector<double> tab((size_t)(p.map + 2) * BSG_STATS_COLUMNS);
                CALL(bsg_recon_statistics(rec, imap, p.resolution, &st, tab.data(), p.map + 2));
                if (imap == 0) printf("Full reconstruction:\n");
                else printf("Half reconstruction %d:\n", imap);
                printf("Friedel symmetry residual:      %.2f\n", st.friedel);
                printf("Coverage:                       %ld (%.2f %%)\n\n", st.coverage, st.coverage_pct);
                if (i != 0) continue;
                printf("Radius\ts(1/A)\tRes(A)\tWeight\tPower\tSignal\tNoise\tSNR\tFSC\n");
                for (int k = 0; k < st.rows && k < p.map + 2; ++k) {
                    const double* t = &tab[(size_t)k * BSG_STATS_COLUMNS];
                    printf("%ld\t%.4f\t%.2f\t%.2f\t%.6f\t%.6f\t%.6f\t%.4f\t%.4f\n", (long)t[0], t[1], t[2], t[3],
                           t[4], t[5], t[6], t[7], t[8]);
                }
                printf("\nResolution estimates:\nSNR(0.5):                       %.4f A\n"
                       "FSC(0.3):                       %.4f A\n\n", st.res_snr, st.res_fsc);
            }
        }
        for (int i = 0; i < p.nmaps; ++i) {
            const int imap = p.nmaps == 2 ? i + 1 : (p.nmaps == 3 ? i : 0);
            const bool want_fom = !o.fom.empty();
            CALL(bsg_recon_finish(rec, imap, vol.data(), want_fom ? fom.data() : nullptr, flags));
            write_mrc_volume(map_name(o.recons, imap), vol.data(), p.map, p.map_sampling, p.map / 2);
            if (want_fom) write_mrc_volume(map_name(o.fom, imap), fom.data(), p.map, p.map_sampling, p.map / 2);
            printf("Writing %s\n", map_name(o.recons, imap).c_str());
        }
        bsg_recon_destroy(rec);
        return 0;
    } catch (const std::exception& e) {
        fprintf(stderr, "breconstruct: %s\n", e.what());
        return 1;
    }
}
