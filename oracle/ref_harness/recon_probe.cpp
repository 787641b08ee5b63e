// recon_probe - test harness linked against the reference library built from
// source (oracle/_ref).  For one particle of a STAR project it runs the
// reference's own per-particle steps (bsoft/src/mg/mg_reconstruct.cpp:150-212)
// and writes the intermediate results as raw little-endian files, so the
// oracle's restatement can be pinned stage by stage:
//   <out>.bkg      double   background value
//   <out>.fft      float[2*ft*ft]  after pad + fft(plan,1)
//   <out>.shift    float[2*ft*ft]  after phase_shift_to_origin
//   <out>.ctf      float[2*ft*ft]  after img_ctf_apply_complex (if ctf_action)
//   <out>.vol      float[2*N^3] + float[N^3] weights: fspace_pack_2D of this particle
// Usage: recon_probe project.star particle_index(0-based) interp ctf_action out_prefix
#include "rwmg.h"
#include "rwimg.h"
#include "mg_processing.h"
#include "mg_reconstruct.h"
#include "mg_ctf.h"
#include "utilities.h"
#include <fstream>

extern int verbose;

static void dump(const std::string& f, const void* p, size_t bytes) {
	std::ofstream o(f, std::ios::binary); o.write((const char*)p, bytes);
}

int main(int argc, char** argv) {
	if ( argc < 6 ) { std::cerr << "usage: recon_probe star idx interp ctf out" << std::endl; return 1; }
	verbose = 0;
	Bstring* files = NULL; string_add(&files, argv[1]);
	Bproject* project = read_project(files);
	long want = atol(argv[2]);
	int interp = atoi(argv[3]), ctf_action = atoi(argv[4]);
	std::string out(argv[5]);
	Vector3<double> sam;
	Vector3<long> size = project_set_reconstruction_size(project, sam, 1, 0);
	Bparticle* part = NULL; Bmicrograph* mg = NULL; long k = 0;
	for ( Bfield* f = project->field; f && !part; f = f->next )
		for ( Bmicrograph* m = f->mg; m && !part; m = m->next )
			for ( Bparticle* p = m->part; p; p = p->next, ++k )
				if ( k == want ) { part = p; mg = m; break; }
	if ( !part ) return 2;
	int ft = part_ft_size(mg->box_size[0] > size[0] ? mg->box_size[0] : size[0], 1, 2);
	double hi_res = sam[0];
	Bimage* prec = new Bimage(Float, TComplex, size, 1);
	prec->sampling(sam);
	prec->check_resolution(hi_res);
	CTFparam em_ctf;
	if ( mg->ctf ) em_ctf.update(mg->ctf);
	Bimage* p = read_img(mg->fpart, 1, part->id - 1);
	p->change_type(Float);
	p->calculate_background();
	double bkg = p->background((long)0);
	dump(out + ".bkg", &bkg, sizeof(double));
	p->sampling(part->pixel_size);
	part->ori[2] = 0;
	p->origin(part->ori);
	if ( part->def > 0 ) em_ctf.defocus_average(part->def);
	double part_weight = 1, pad_ratio = ft*1.0L/p->sizeX();
	if ( pad_ratio > 1 ) { pad_ratio *= pad_ratio*0.6; part_weight /= pad_ratio; p->pad(ft, FILL_BACKGROUND); }
	fft_plan plan = fft_setup_plan(ft, ft, 1, FFTW_FORWARD, 1);
	p->fft(plan, 1);
	dump(out + ".fft", p->data_pointer(), sizeof(float)*2*ft*ft);
	p->phase_shift_to_origin();
	dump(out + ".shift", p->data_pointer(), sizeof(float)*2*ft*ft);
	if ( ctf_action ) {
		double wiener = ctf_action > 2 ? 0.2 : 0;
		img_ctf_apply_complex(p, em_ctf, (ctf_action==1), wiener, 0, hi_res);
		dump(out + ".ctf", p->data_pointer(), sizeof(float)*2*ft*ft);
	}
	Vector3<double> part_scale(1,1,1);
	prec->fspace_pack_2D(p, part->view.matrix(), hi_res, 0, part_scale, 0, part_weight, interp);
	long N3 = size.volume();
	dump(out + ".vol", prec->data_pointer(), sizeof(float)*2*N3);
	dump(out + ".w", prec->next->next->data_pointer(), sizeof(float)*N3);
	std::cout << "ft " << ft << " hi_res " << hi_res << " bkg " << bkg << " origin " << part->ori
		<< " weight " << part_weight << " view " << part->view << " id " << part->id << " def " << part->def << " pix " << part->pixel_size << std::endl;
	fft_destroy_plan(plan);
	return 0;
}
