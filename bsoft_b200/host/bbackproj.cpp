// bbackproj - drop-in for the reference's bbackproj (bsoft/src/bbackproj.cpp)
// over libbsgpu's real-space back-projection (bsg_backproj_*).
//
// Reads the STAR project(s), resolves what project_back_projection
// (bsoft/src/mg/mg_reconstruct.cpp:1524-1624) takes from them — the map size
// and sampling (project_set_reconstruction_size, :596-651), each selected
// particle's origin (a coordinate <= 0 falls back to the image file's origin,
// then to the map's, per axis), view, magnification over the scale, pixel size,
// and the half-map index of the round-robin partial maps — streams the particle
// images through the GPU and writes the map(s) as bbackproj names them
// (bbackproj.cpp:214-232: out.mrc, out_01.mrc / out_02.mrc for half maps).
//
// The reference plans its image transforms at the map's x, y size
// (bbackproj.cpp:170-171) although Bimage::fft needs a plan of the image's size
// (Bimage_fft.cpp:173); the two agree when the map edge is the image edge
// (scale 1, no -size), and this program transforms at the image size always.
//
// Usage: bbackproj [options] input.star [input.star ...]
#include "bsgpu.h"
#include "project.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

using namespace bsh;

namespace {

struct Options {
    double resolution = 0, sampling = 0, scale = 1;
    int size = 0, nmaps = 0, threads = 1, batch = 256, device = 0;
    double rescale_avg = 0, rescale_std = 0;
    std::string symmetry = "C1";
    std::string recons;
    bool plan_only = false;
    std::vector<std::string> inputs;
};

struct Plan {
    int n = 0, map = 0, nmaps = 1;
    double map_sampling = 0, pixel = 0;
    std::vector<double> rec;                  // BSG_BACKPROJ_DOUBLES per particle
    std::vector<std::pair<int, long>> src;    // (micrograph, image index)
};

Plan plan_backprojection(const std::vector<Micrograph>& mgs, const Options& o) {
    int first = -1;
    for (size_t i = 0; i < mgs.size(); ++i)
        if (!mgs[i].part_id.empty()) { first = (int)i; break; }
    if (first < 0) throw std::runtime_error("no particles");
    const Micrograph& m0 = mgs[first];
    const StackHeader h0 = read_stack_header(m0.particle_file);
    double sam = o.sampling;
    if (sam < 0.1) sam = m0.pixel[0] > 0 ? m0.pixel[0] : 0.0;
    if (sam < 0.1) sam = m0.pixel_size;
    if (sam < 0.1) sam = h0.sampling(0);
    Plan p;
    p.n = h0.nx();
    p.map = o.size ? o.size : std::max(1, (int)(h0.nx() * o.scale));
    p.map_sampling = sam / o.scale;
    p.nmaps = o.nmaps < 1 ? 1 : (o.nmaps > 3 ? 3 : o.nmaps);
    const double mo = (double)(p.map / 2);    // Bimage::default_origin
    int t = std::max(1, o.threads);
    if ((p.nmaps & 2) && (t % 2)) ++t;
    long k = 0;
    for (size_t mi = 0; mi < mgs.size(); ++mi) {
        const Micrograph& mg = mgs[mi];
        if (mg.part_id.empty()) continue;
        const StackHeader h = read_stack_header(mg.particle_file);
        for (size_t i = 0; i < mg.part_id.size(); ++i) {
            if (mg.select[i] <= 0) continue;
            double r[BSG_BACKPROJ_DOUBLES] = {};
            const double fo[2] = {h.image_origin(0, mg.part_id[i] - 1), h.image_origin(1, mg.part_id[i] - 1)};
            r[0] = mg.ox[i] > 0 ? mg.ox[i] : (fo[0] > 0 ? fo[0] : mo);
            r[1] = mg.oy[i] > 0 ? mg.oy[i] : (fo[1] > 0 ? fo[1] : mo);
            view_matrix(mg.vx[i], mg.vy[i], mg.vz[i], mg.va[i], r + 2);
            r[11] = (mg.mag[i] > 0 ? mg.mag[i] : 1.0) / o.scale;     // Bparticle's default magnification is 1
            r[12] = (p.nmaps & 2) ? (double)((k % t) % 2) : 0.0;    // even partial maps form half 1
            r[13] = mg.pixel[i] > 0 ? mg.pixel[i] : h.sampling(0);
            p.rec.insert(p.rec.end(), r, r + BSG_BACKPROJ_DOUBLES);
            p.src.push_back({(int)mi, mg.part_id[i] - 1});
            ++k;
        }
    }
    p.pixel = p.rec.empty() ? sam : p.rec[13];
    return p;
}

void usage() {
    fprintf(stderr,
            "Usage: bbackproj [options] input.star [input.star]\n"
            "  -resolution 3.4  -size 120  -sampling 2  -scale 1  -symmetry D6  -rescale avg,std\n"
            "  -fullmap  -halfmaps  -threads 2  -reconstruction out.mrc  -batch 256  -device 0  -plan\n");
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
        if (a == "-resolution") o.resolution = atof(val().c_str());
        else if (a == "-size") o.size = atoi(val().c_str());
        else if (a == "-sampling") o.sampling = atof(val().c_str());
        else if (a == "-scale") {
            o.scale = atof(val().c_str());
            if (o.scale < 0.0001) throw std::runtime_error("-scale: a scale must be specified");
        }
        else if (a == "-fullmap") o.nmaps += 1;
        else if (a == "-halfmaps") o.nmaps += 2;
        else if (a == "-threads") o.threads = atoi(val().c_str());
        else if (a == "-symmetry" || a == "-sym") o.symmetry = val();
        else if (a == "-rescale") {
            const std::string v = val();
            const size_t c = v.find(',');
            if (c == std::string::npos) throw std::runtime_error("-rescale: both average and standard deviation must be given");
            o.rescale_avg = atof(v.c_str());
            o.rescale_std = atof(v.c_str() + c + 1);
            if (!(o.rescale_std > 0)) throw std::runtime_error("-rescale: a positive standard deviation must be given");
        }
        else if (a == "-reconstruction" || a == "-recon") o.recons = val();
        else if (a == "-batch") o.batch = atoi(val().c_str());
        else if (a == "-device") o.device = atoi(val().c_str());
        else if (a == "-plan") o.plan_only = true;
        else if (a == "-edge" || a == "-classes" || a == "-datatype" || a == "-output")
            throw std::runtime_error("option " + a + " is not supported by this drop-in");
        else if (a == "-verbose") (void)val();
        else if (a == "-h" || a == "-help") { usage(); exit(0); }
        else if (a[0] == '-') throw std::runtime_error("unknown option " + a);
        else o.inputs.push_back(a);
    }
    if (o.inputs.empty()) throw std::runtime_error("no parameter files specified");
    return o;
}

std::string map_name(const std::string& base, int imap) {
    if (!imap) return base;
    const size_t dot = base.find_last_of('.');
    char tag[16];
    snprintf(tag, sizeof(tag), "_%02d", imap);
    if (dot == std::string::npos) return base + tag;
    return base.substr(0, dot) + tag + base.substr(dot);
}

#define CALL(x)                                                                                   \
    do {                                                                                          \
        if ((x) != BSG_OK) throw std::runtime_error(std::string(#x) + ": " + bsg_last_error());   \
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
        const Plan p = plan_backprojection(mgs, o);
        const long np = (long)p.src.size();
        if (o.plan_only) {
            printf("n %d map %d map_sampling %.17g pixel %.17g nmaps %d particles %ld\n", p.n, p.map,
                   p.map_sampling, p.pixel, p.nmaps, np);
            for (long i = 0; i < np; ++i)
                for (int j = 0; j < BSG_BACKPROJ_DOUBLES; ++j)
                    printf("%.17g%c", p.rec[i * BSG_BACKPROJ_DOUBLES + j], j + 1 < BSG_BACKPROJ_DOUBLES ? ' ' : '\n');
            return 0;
        }
        if (o.recons.empty()) throw std::runtime_error("no -reconstruction file name given");
        bsg_backproj_config cfg = {};
        cfg.n = p.n; cfg.map = p.map; cfg.pixel = p.pixel; cfg.resolution = o.resolution;
        cfg.nmaps = p.nmaps; cfg.batch = o.batch; cfg.device = o.device;
        bsg_backproj* bp = nullptr;
        CALL(bsg_backproj_create(&cfg, &bp));
        if (o.symmetry != "C1" && !o.symmetry.empty()) {
            std::vector<double> ax;
            std::vector<int> ord;
            for (const SymOp& g : symmetry_generators(o.symmetry)) {
                ax.insert(ax.end(), g.a, g.a + 3);
                ord.push_back(g.order);
            }
            CALL(bsg_backproj_set_symmetrize(bp, ax.data(), ord.data(), (int)ord.size()));
        }
        if (o.rescale_std > 0) CALL(bsg_backproj_set_rescale(bp, o.rescale_avg, o.rescale_std));
        const long n2 = (long)p.n * p.n;
        const long B = std::max(1, o.batch);
        std::vector<float> buf((size_t)(B * n2));
        std::map<int, StackHeader> hdrs;
        for (long b0 = 0; b0 < np; b0 += B) {
            const long cnt = std::min(B, np - b0);
            for (long i = 0; i < cnt; ++i) {
                const auto& s = p.src[b0 + i];
                const Micrograph& mg = mgs[s.first];
                if (!hdrs.count(s.first)) hdrs[s.first] = read_stack_header(mg.particle_file);
                const StackHeader& h = hdrs[s.first];
                if (h.nx() != p.n || h.ny() != p.n)
                    throw std::runtime_error(mg.particle_file + ": images must all be " + std::to_string(p.n) + "^2");
                read_stack_images(mg.particle_file, h, s.second, 1, buf.data() + i * n2);
            }
            CALL(bsg_backproj_add(bp, buf.data(), p.rec.data() + b0 * BSG_BACKPROJ_DOUBLES, cnt, 0));
        }
        const size_t n3 = (size_t)p.map * p.map * p.map;
        std::vector<float> vol(n3);
        // bbackproj's output maps: the full map, the two half maps, or all three
        std::vector<int> maps;
        if (p.nmaps & 1) maps.push_back(0);
        if (p.nmaps & 2) { maps.push_back(1); maps.push_back(2); }
        for (int imap : maps) {
            CALL(bsg_backproj_finish(bp, imap, vol.data(), 0));
            write_mrc_volume(map_name(o.recons, imap), vol.data(), p.map, p.map_sampling, p.map / 2);
            printf("Writing %s\n", map_name(o.recons, imap).c_str());
        }
        bsg_backproj_destroy(bp);
        return 0;
    } catch (const std::exception& e) {
        fprintf(stderr, "bbackproj: %s\n", e.what());
        return 1;
    }
}
