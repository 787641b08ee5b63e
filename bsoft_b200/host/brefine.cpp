// brefine - drop-in for the reference's brefine (bsoft/src/brefine.cpp) grid
// refinement on one B200: reads the STAR project, the particle stacks and
// the reference map, refines every selected particle's view and origin (and
// its defocus with -defocus) by img_refine_grid through libbsgpu's
// bsg_match_refine (include/bsgpu.h), and writes the project with the new
// parameters and figures of merit.
//
// Options (the reference's spelling, brefine.cpp:23-67):
//   -reference map.mrc        reference map (required)
//   -grid 2.5,0.3             angular step and accuracy (degrees; required)
//   -step 0.4,0.1             origin step and accuracy (pixels; default 0.4,0.1)
//   -defocus 0.002            defocus search step (micrometres below 10, else angstrom)
//   -resolution 20[,250]      high (and low) resolution limits (angstrom)
//   -kernel 8,2               FSI kernel width and power
//   -contrast                 invert the contrast
//   -select 14   -all         particle selection
//   -output out.star          output project
//   -batch 4096  -device 0
//   -fomtype frc|dpr          figure of merit (brefine.cpp:124-127: the first letter decides)
//   -magnification 0.01       magnification search: per-axis pixel-size factors 1 +- m
//                             (img_refine_grid's second stage); the refined pixel
//                             sizes x, y are written with the particle
// Not supported (rejected): -monte, -symmetry, -mask, -FSC, -edge.
//
// Flow as project_refine_orientations / part_refine_orientation
// (bsoft/src/mg/mg_refine.cpp:249-457, 491-648): one reference preparation,
// particles of one stack prepared together (each stack is normalised with
// its own header statistics, rwMRC.cpp:181-184), the figure of merit and
// its cross-validation value stored with the particle.
#include "bsgpu.h"
#include "project.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace {

using namespace bsh;

struct Options {
    std::string reference, output;
    double alpha = 0, accuracy = 0.5 * M_PI / 180.0;   // radians (brefine.cpp:80)
    double shift_step = 0.4, shift_accuracy = 0.1;
    double def_std = 0, hi_res = 0, lo_res = 0, max_mag = 0;
    int kernel_w = 8, kernel_p = 2, select = -1, batch = 4096, device = 0, fom_type = 0;
    bool contrast = false, all = false;
    std::vector<std::string> inputs;
};

// "a,b" -> values (Boption::values)
int values(const std::string& s, double& a, double& b) {
    const size_t c = s.find(',');
    a = atof(s.c_str());
    if (c == std::string::npos) return 1;
    b = atof(s.c_str() + c + 1);
    return 2;
}

Options parse(int argc, char** argv) {
    Options o;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto val = [&]() -> std::string {
            if (i + 1 >= argc) throw std::runtime_error("option " + a + " needs a value");
            return argv[++i];
        };
        if (a == "-reference") o.reference = val();
        else if (a == "-output") o.output = val();
        else if (a == "-grid") {
            double s = 0, acc = 0.5;
            values(val(), s, acc);
            o.alpha = s * M_PI / 180.0;       // brefine.cpp:117-121
            o.accuracy = acc * M_PI / 180.0;
        } else if (a == "-step") values(val(), o.shift_step, o.shift_accuracy);
        else if (a == "-defocus") {
            o.def_std = atof(val().c_str());
            if (o.def_std < 10) o.def_std *= 1e4;   // micrometres given (brefine.cpp:140-145)
        } else if (a == "-resolution") {
            values(val(), o.hi_res, o.lo_res);
            if (o.lo_res > 0 && o.lo_res < o.hi_res) std::swap(o.hi_res, o.lo_res);
        } else if (a == "-kernel") {
            double w = 8, p = 2;
            values(val(), w, p);
            o.kernel_w = (int)w;
            o.kernel_p = (int)p;
        } else if (a == "-fomtype") {
            const std::string v = val();
            if (!v.empty() && v[0] == 'f') o.fom_type = 0;
            if (!v.empty() && v[0] == 'd') o.fom_type = 1;
        } else if (a == "-magnification") {
            o.max_mag = atof(val().c_str());
            if (o.max_mag < 0) throw std::runtime_error("-magnification: a maximum magnification adjustment must be specified");
        } else if (a == "-contrast") o.contrast = true;
        else if (a == "-select") o.select = atoi(val().c_str());
        else if (a == "-all") o.all = true;
        else if (a == "-batch") o.batch = atoi(val().c_str());
        else if (a == "-device") o.device = atoi(val().c_str());
        else if (a[0] == '-') throw std::runtime_error("unknown or unsupported option " + a);
        else o.inputs.push_back(a);
    }
    if (o.inputs.empty()) throw std::runtime_error("no parameter file given");
    if (o.reference.empty()) throw std::runtime_error("no -reference map given");
    if (!(o.alpha > 0)) throw std::runtime_error("-grid step,accuracy (degrees) is required");
    return o;
}

#define CALL(x)                                                                                 \
    do {                                                                                        \
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
        if (o.all)
            for (auto& mg : mgs)
                for (auto& s : mg.select) s = 1;
        const MrcHeader mh = read_mrc_header(o.reference);
        if (mh.nx != mh.ny || mh.nx != mh.nz) throw std::runtime_error(o.reference + ": the map must be cubic");
        const std::vector<float> map = read_mrc_volume(o.reference, mh);
        const double map_origin[3] = {mh.image_origin(0), mh.image_origin(1), mh.image_origin(2)};
        int first = -1;
        for (size_t i = 0; i < mgs.size(); ++i)
            if (!mgs[i].part_id.empty()) { first = (int)i; break; }
        if (first < 0) throw std::runtime_error("no particles");
        const StackHeader h0 = read_stack_header(mgs[first].particle_file);
        bsg_match_config cfg = {};
        cfg.n = h0.nx();
        cfg.map = mh.nx;
        cfg.map_sampling = mh.sampling(0);
        cfg.pixel = mgs[first].pixel[0] > 0 ? mgs[first].pixel[0] : h0.sampling(0);
        cfg.hi_res = o.hi_res;
        cfg.lo_res = o.lo_res;
        cfg.kernel_width = o.kernel_w;
        cfg.kernel_power = o.kernel_p;
        cfg.device = o.device;
        bsg_match* m = nullptr;
        CALL(bsg_match_create(&cfg, &m));
        CALL(bsg_match_set_reference(m, map.data(), map_origin, 0));
        const long n2 = (long)h0.nx() * h0.ny();
        std::vector<std::vector<double>> fom(mgs.size()), fcv(mgs.size());
        long done = 0;
        Ctf em;
        for (size_t mi = 0; mi < mgs.size(); ++mi) {
            Micrograph& mg = mgs[mi];
            fom[mi].assign(mg.part_id.size(), 0.0);
            fcv[mi].assign(mg.part_id.size(), 0.0);
            if (mg.has_ctf) em = mg.ctf;
            std::vector<long> sel;
            for (size_t i = 0; i < mg.part_id.size(); ++i)
                if (o.select >= 0 ? mg.select[i] == o.select : mg.select[i] > 0) sel.push_back((long)i);
            if (sel.empty()) continue;
            const StackHeader h = read_stack_header(mg.particle_file);
            if (h.nx() != cfg.n || h.ny() != cfg.n) throw std::runtime_error(mg.particle_file + ": particle size differs");
            for (size_t b0 = 0; b0 < sel.size(); b0 += (size_t)std::max(1, o.batch)) {
                const size_t cnt = std::min(sel.size() - b0, (size_t)std::max(1, o.batch));
                std::vector<float> imgs(cnt * n2);
                std::vector<double> ctf(cnt * BSG_MATCH_CTF_DOUBLES, 0.0), start(cnt * BSG_MATCH_REFINE_START_DOUBLES);
                for (size_t j = 0; j < cnt; ++j) {
                    const long i = sel[b0 + j];
                    read_stack_images(mg.particle_file, h, mg.part_id[i] - 1, 1, imgs.data() + j * n2);
                    // the particle's CTF: the micrograph's, at the particle's
                    // defocus when it has one (part_refine_orientation :567-598)
                    Ctf c = em;
                    if (mg.defocus[i] > 1) c.defocus = mg.defocus[i];
                    double co[7];
                    c.coefficients(co);
                    double* r = &ctf[j * BSG_MATCH_CTF_DOUBLES];
                    r[0] = c.volt;
                    for (int k = 0; k < 5; ++k) r[1 + k] = co[k];
                    r[6] = (o.def_std > 0 ? BSG_MATCH_APPLY_CTF : 0) | (o.contrast ? BSG_MATCH_INVERT : 0);
                    double* s = &start[j * BSG_MATCH_REFINE_START_DOUBLES];
                    s[0] = (double)j;
                    s[1] = mg.vx[i]; s[2] = mg.vy[i]; s[3] = mg.vz[i]; s[4] = mg.va[i];
                    s[5] = mg.ox[i]; s[6] = mg.oy[i];
                }
                CALL(bsg_match_set_images(m, imgs.data(), (long)cnt, ctf.data(), h.mean(), h.stddev(), 0));
                std::vector<double> out(cnt * BSG_MATCH_REFINE_RESULT_DOUBLES);
                CALL(bsg_match_refine(m, start.data(), (long)cnt, o.alpha, o.accuracy, o.shift_step, o.shift_accuracy,
                                      o.def_std, o.max_mag, out.data(), o.fom_type == 1 ? BSG_MATCH_SCORE_DPR : 0));
                for (size_t j = 0; j < cnt; ++j) {
                    const long i = sel[b0 + j];
                    const double* r = &out[j * BSG_MATCH_REFINE_RESULT_DOUBLES];
                    mg.vx[i] = r[0]; mg.vy[i] = r[1]; mg.vz[i] = r[2]; mg.va[i] = r[3];
                    mg.ox[i] = r[4]; mg.oy[i] = r[5];
                    fom[mi][i] = r[6];
                    fcv[mi][i] = r[7];
                    if (o.def_std > 0 && r[9] > 1) mg.defocus[i] = r[9];
                    if (o.max_mag > 0) {
                        mg.pixel[i] = r[10];
                        mg.pixel_y[i] = r[11];
                    }
                }
                done += (long)cnt;
            }
        }
        bsg_match_destroy(m);
        if (!o.output.empty()) write_project(o.output, mgs, fom, fcv);
        printf("Refined %ld particles\n", done);
        return 0;
    } catch (const std::exception& e) {
        fprintf(stderr, "brefine: %s\n", e.what());
        return 1;
    }
}
