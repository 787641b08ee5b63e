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
//                             (img_refine_grid's second stage, or img_refine_monte's
//                             random factors); the refined pixel sizes x, y are
//                             written with the particle
//   -monte 80                 Monte Carlo refinement (img_refine_monte) with
//   -shift 0.5 -view 0.02 -angle 2   its origin, view and angle steps, and
//   -seed 1                   the random() seed (default: the process id, as the
//                             reference seeds it)
//   -symmetry D2              refine from every symmetry-related view of each particle
//                             (symmetry_get_all_views) and keep the best
// Not supported (rejected): -mask, -FSC, -edge.
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

#include <unistd.h>

namespace {

using namespace bsh;

struct Options {
    std::string reference, output;
    double alpha = 0, accuracy = 0.5 * M_PI / 180.0;   // radians (brefine.cpp:80)
    double shift_step = 0.4, shift_accuracy = 0.1;
    double def_std = 0, hi_res = 0, lo_res = 0, max_mag = 0;
    int max_iter = 0;                                   // -monte
    double shift_std = 0.1, view_std = 0.01, max_angle = M_PI / 360;   // brefine.cpp:85-87
    long seed = -1;
    std::string symmetry = "C1";
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
        } else if (a == "-monte") {
            o.max_iter = atoi(val().c_str());
            if (o.max_iter < 1) throw std::runtime_error("-monte: a number of iterations must be specified");
        } else if (a == "-shift") {
            o.shift_std = atof(val().c_str());
            if (o.shift_std < 0.001) throw std::runtime_error("-shift: an origin shift standard deviation must be specified");
        } else if (a == "-view") {
            o.view_std = atof(val().c_str());
            if (o.view_std < 0.001) throw std::runtime_error("-view: a view shift standard deviation must be specified");
        } else if (a == "-angle") {
            o.max_angle = atof(val().c_str());
            if (o.max_angle < 0.1) throw std::runtime_error("-angle: a maximum rotation angle adjustment must be specified");
            o.max_angle *= M_PI / 180.0;
        } else if (a == "-symmetry" || a == "-sym") {
            o.symmetry = val();
        } else if (a == "-seed") {
            o.seed = atol(val().c_str());
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
    if (!(o.alpha > 0) && o.max_iter < 1) throw std::runtime_error("-grid step,accuracy (degrees) or -monte is required");
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
        {
            // project_refine_orientations' weight curve when none is given:
            // C_curve(diam, 1 / real size of the cut map) (mg_refine.cpp:366-367,
            // bsoft/src/util/ctf.cpp:795-810)
            bsg_match_info_t info;
            CALL(bsg_match_info(m, &info));
            const double fstep = 1.0 / (info.diam * info.map_sampling_cut);
            std::vector<double> w(info.diam);
            for (int i = 0; i < info.diam; ++i) {
                double s2 = i * fstep;
                s2 *= s2;
                w[i] = 0.893 * exp(-0.2465 * s2) + 0.2563 * exp(-1.7100 * s2) + 0.7570 * exp(-6.4094 * s2) +
                       1.0487 * exp(-18.6113 * s2) + 0.3575 * exp(-50.2523 * s2);
            }
            CALL(bsg_match_set_shell_weights(m, w.data(), (int)w.size()));
        }
        const long n2 = (long)h0.nx() * h0.ny();
        std::vector<std::vector<double>> fom(mgs.size()), fcv(mgs.size());
        long done = 0;
        bool seeded = false;
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
                // part_refine_orientation refines from every view of
                // symmetry_get_all_views (mg_refine.cpp:584-621): nsym records per particle
                const size_t nsym = symmetry_views(o.symmetry, 0, 0, 1, 0).size();
                std::vector<double> ctf(cnt * BSG_MATCH_CTF_DOUBLES, 0.0), start(cnt * nsym * BSG_MATCH_REFINE_START_DOUBLES);
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
                    const std::vector<RefView> views = symmetry_views(o.symmetry, mg.vx[i], mg.vy[i], mg.vz[i], mg.va[i]);
                    for (size_t k = 0; k < nsym; ++k) {
                        double* s = &start[(j * nsym + k) * BSG_MATCH_REFINE_START_DOUBLES];
                        s[0] = (double)j;
                        s[1] = views[k].v[0]; s[2] = views[k].v[1]; s[3] = views[k].v[2]; s[4] = views[k].a;
                        s[5] = mg.ox[i]; s[6] = mg.oy[i];
                    }
                }
                CALL(bsg_match_set_images(m, imgs.data(), (long)cnt, ctf.data(), h.mean(), h.stddev(), 0));
                std::vector<double> out(cnt * nsym * BSG_MATCH_REFINE_RESULT_DOUBLES);
                const long nrec = (long)(cnt * nsym);
                const int fflags = o.fom_type == 1 ? BSG_MATCH_SCORE_DPR : 0;
                // one random() stream over the run: seeded on the first batch
                // (srandom(getpid()) in the reference), continued after
                auto seed_for_batch = [&]() -> unsigned long long {
                    if (seeded) return 0ULL;
                    seeded = true;
                    const unsigned long long sd = o.seed >= 0 ? (unsigned long long)o.seed : (unsigned long long)getpid();
                    return sd != 0 ? sd : 1ULL;
                };
                if (o.max_iter > 0)
                    CALL(bsg_match_refine_monte(m, start.data(), nrec, o.max_iter, o.def_std, o.shift_std,
                                                o.view_std, o.max_angle, o.max_mag, seed_for_batch(), out.data(), fflags));
                else
                    CALL(bsg_match_refine(m, start.data(), nrec, o.alpha, o.accuracy, o.shift_step, o.shift_accuracy,
                                          o.def_std, o.max_mag, out.data(), fflags));
                for (size_t j = 0; j < cnt; ++j) {
                    const long i = sel[b0 + j];
                    // part_refine_orientation keeps, in view order, a result whose figure
                    // of merit exceeds the best so far, starting from 0 (mg_refine.cpp:532,
                    // 609-620), and numbers the winning symmetry view in the selection
                    double best = 0;
                    for (size_t k = 0; k < nsym; ++k) {
                        const double* r = &out[(j * nsym + k) * BSG_MATCH_REFINE_RESULT_DOUBLES];
                        if (!(best < r[6])) continue;
                        best = r[6];
                        mg.select[i] = (long)k + 1;
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
