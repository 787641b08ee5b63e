// stage_probe - per-stage CPU time of the reference's particle_reconstruct
// loop (bsoft/src/mg/mg_reconstruct.cpp:143-229), single-threaded, over the
// first `count` particles of a STAR project.  Test and measurement
// infrastructure only: it links the reference library compiled from source
// (oracle/_ref) and times the reference's own calls, in the reference's
// order, with a steady clock around each:
//   read      read_img + change_type
//   background calculate_background
//   pad       pad(ft, FILL_BACKGROUND)
//   fft       fft(plan, 1)   (FFTW3-API stand-in: oracle/fftw3_standin)
//   shift     phase_shift_to_origin
//   ctf       img_ctf_apply_complex (flip)
//   pack      fspace_pack_2D (trilinear)
// Prints one line "stage seconds" per stage and the particle count.
// Usage: stage_probe project.star count
#include "rwmg.h"
#include "rwimg.h"
#include "mg_processing.h"
#include "mg_reconstruct.h"
#include "mg_ctf.h"
#include "utilities.h"

#include <chrono>
#include <cstdio>

extern int verbose;

namespace {
using clk = std::chrono::steady_clock;
double since(clk::time_point& t) {
    const clk::time_point n = clk::now();
    const double s = std::chrono::duration<double>(n - t).count();
    t = n;
    return s;
}
}  // namespace

int main(int argc, char** argv) {
    if ( argc < 3 ) { std::cerr << "usage: stage_probe project.star count" << std::endl; return 1; }
    verbose = 0;
    Bstring* files = NULL; string_add(&files, argv[1]);
    Bproject* project = read_project(files);
    const long count = atol(argv[2]);
    Vector3<double> sam;
    Vector3<long> size = project_set_reconstruction_size(project, sam, 1, 0);
    Bmicrograph* mg0 = project->field->mg;
    const int ft = part_ft_size(mg0->box_size[0] > size[0] ? mg0->box_size[0] : size[0], 1, 2);
    double hi_res = sam[0];
    Bimage* prec = new Bimage(Float, TComplex, size, 1);
    prec->sampling(sam);
    prec->check_resolution(hi_res);
    fft_plan plan = fft_setup_plan(ft, ft, 1, FFTW_FORWARD, 1);
    CTFparam em_ctf;
    double t_read = 0, t_bkg = 0, t_pad = 0, t_fft = 0, t_shift = 0, t_ctf = 0, t_pack = 0;
    long done = 0;
    for ( Bfield* f = project->field; f && done < count; f = f->next )
        for ( Bmicrograph* mg = f->mg; mg && done < count; mg = mg->next )
            for ( Bparticle* part = mg->part; part && done < count; part = part->next ) {
                if ( mg->ctf ) em_ctf.update(mg->ctf);
                clk::time_point t = clk::now();
                Bimage* p = read_img(mg->fpart, 1, part->id - 1);
                if ( !p ) return 2;
                p->change_type(Float);
                t_read += since(t);
                p->calculate_background();
                t_bkg += since(t);
                p->sampling(part->pixel_size);
                part->ori[2] = 0;
                p->origin(part->ori);
                if ( part->def > 0 ) em_ctf.defocus_average(part->def);
                Vector3<double> part_scale(1, 1, 1);
                if ( part->mag > 0 ) part_scale /= part->mag;
                double part_weight = 1, pad_ratio = ft * 1.0L / p->sizeX();
                t = clk::now();
                if ( pad_ratio > 1 ) { pad_ratio *= pad_ratio * 0.6; part_weight /= pad_ratio; p->pad(ft, FILL_BACKGROUND); }
                t_pad += since(t);
                p->fft(plan, 1);
                t_fft += since(t);
                p->phase_shift_to_origin();
                t_shift += since(t);
                img_ctf_apply_complex(p, em_ctf, 1, 0, 0, hi_res);
                t_ctf += since(t);
                prec->fspace_pack_2D(p, part->view.matrix(), hi_res, 0, part_scale, 0, part_weight, 2);
                t_pack += since(t);
                if ( mg->ctf ) em_ctf.defocus_average(mg->ctf->defocus_average());
                delete p;
                ++done;
            }
    printf("particles %ld\nft %d\nread %.6f\nbackground %.6f\npad %.6f\nfft %.6f\nshift %.6f\nctf %.6f\npack %.6f\n",
           done, ft, t_read, t_bkg, t_pad, t_fft, t_shift, t_ctf, t_pack);
    fft_destroy_plan(plan);
    delete prec;
    return done == count ? 0 : 3;
}
