// refine_probe - test harness linked against the reference library built
// from source (oracle/_ref): brefine's grid refinement of particles against a
// map, one particle at a time, through the reference's own functions:
// the map and particle preparation of project_refine_orientations /
// part_refine_orientation (bsoft/src/mg/mg_refine.cpp:279-365, 509-563) and
// img_refine_grid (:1086-1195, with img_fit_in_recip_space_grid :862-950).
// Prints per particle: view x y z angle, origin x y (pixels of the uncut
// image), figure of merit, cross-validation figure, hypotheses scored,
// defocus after refinement (angstrom).
// Usage:
//   refine_probe map.mrc stack.mrc pixel hi_res start.txt ctf.txt alpha_step_deg accuracy_deg shift_step shift_accuracy
//                [verbose [def_std [fom_type [max_mag [c_curve [max_iter shift_std view_std max_angle_deg seed]]]]]]
// start.txt: "x y z angle(rad) origin_x origin_y" per particle; ctf.txt as
// for match_probe ("volt abw00 abw20 abw22 abw2m2 abw40 apply").  def_std > 0
// turns on the defocus search with the CTF applied, as brefine -defocus does
// (part_refine_orientation, mg_refine.cpp:569-576).  Without it the CTF must
// not be applied: the reference's defocus loop would not end (def += 0).
#include "rwimg.h"
#include "mg_processing.h"
#include "Bimage.h"
#include "FSI_Kernel.h"
#include "ctf.h"
#include "View.h"
#include "utilities.h"
#include <cstdio>
#include <fstream>
#include <sstream>

extern int verbose;

// external linkage in the reference, declared in no header (mg_refine.cpp:34-38)
double img_refine_grid(Bimage* p, Bimage* pref, double hi_res, double lo_res, int flags,
                       double alpha_step, double accuracy, double shift_step,
                       double shift_accuracy, double max_mag, int fom_type, vector<double>& weight,
                       CTFparam* em_ctf, double def_std, FSI_Kernel* kernel, long &number);
double img_refine_monte(Bimage* p, Bimage* pref, double hi_res, double lo_res, int flags,
                        int max_iter, int fom_type, vector<double>& weight, CTFparam* em_ctf,
                        double def_std, double shift_std, double view_std,
                        double max_angle, double max_mag, FSI_Kernel* kernel, long &number);
extern int randseed;

int main(int argc, char** argv) {
	if ( argc < 11 ) { fprintf(stderr, "usage: refine_probe map stack pixel hi_res start ctf alpha acc step step_acc"
		" [verbose [def_std [fom_type [max_mag [c_curve]]]]]\n"); return 1; }
	verbose = argc > 11 ? atoi(argv[11]) : 0;
	double def_std = argc > 12 ? atof(argv[12]) : 0;
	int fom_type = argc > 13 ? atoi(argv[13]) : 0;        // 1: DPR (brefine -fomtype dpr)
	double max_mag = argc > 14 ? atof(argv[14]) : 0;      // brefine -magnification
	int c_curve = argc > 15 ? atoi(argv[15]) : 0;         // 1: brefine's weight curve
	// brefine -monte: img_refine_monte with max_iter iterations, the shift,
	// view and angle steps, and random() seeded with `seed` once before the
	// first particle (project_refine_orientations seeds it with getpid(),
	// mg_refine.cpp:276; the particles then draw one after another)
	int max_iter = argc > 16 ? atoi(argv[16]) : 0;
	double shift_std = argc > 17 ? atof(argv[17]) : 0;
	double view_std = argc > 18 ? atof(argv[18]) : 0;
	double max_angle = argc > 19 ? atof(argv[19])*M_PI/180.0 : 0;
	if ( max_iter > 0 ) {
		srandom((unsigned) (argc > 20 ? atol(argv[20]) : 1));
		randseed = 1;
	}
	double pixel = atof(argv[3]), hi_res = atof(argv[4]);
	double alpha_step = atof(argv[7])*M_PI/180.0, accuracy = atof(argv[8])*M_PI/180.0;
	double shift_step = atof(argv[9]), shift_accuracy = atof(argv[10]);

	Bimage* pref = read_img(argv[1], 1, -1);
	if ( !pref ) return 2;
	pref->check_resolution(hi_res);
	if ( pref->compound_type() == TSimple ) pref->fft();
	int diam = (int) (2.2*pref->real_size()[0]/hi_res + 0.5);
	if ( diam%2 ) diam += 1;
	Vector3<long> size(diam, diam, diam);
	if ( diam < pref->sizeX() ) pref->change_transform_size(size);
	pref->set(0, 0);
	pref->set(1, 0);
	pref->check_resolution(hi_res);
	FSI_Kernel* kernel = new FSI_Kernel(8, 2);
	pref->phase_shift_to_origin();

	std::vector<std::vector<double>> start, ctfs;
	{ std::ifstream f(argv[5]); std::string line;
	  while ( std::getline(f, line) ) { std::istringstream s(line); std::vector<double> v; double t;
	    while ( s >> t ) v.push_back(t); if ( v.size() >= 6 ) start.push_back(v); } }
	{ std::ifstream f(argv[6]); std::string line;
	  while ( std::getline(f, line) ) { std::istringstream s(line); std::vector<double> v; double t;
	    while ( s >> t ) v.push_back(t); if ( v.size() >= 7 ) ctfs.push_back(v); } }

	// project_refine_orientations weighs the shells with C_curve unless a
	// curve is given (mg_refine.cpp:366-367); 0 keeps img_recip_space_fom's
	// unit weights
	vector<double> weight;
	if ( c_curve ) weight = C_curve(pref->sizeX(), 1/pref->real_size()[0]);
	for ( size_t i = 0; i < start.size() && i < ctfs.size(); ++i ) {
		Bimage* p = read_img(argv[2], 1, (long)i);
		if ( !p ) return 3;
		p->sampling(pixel, pixel, 1);
		p->origin(Vector3<double>(start[i][4], start[i][5], 0));
		p->change_type(Float);
		p->rescale_to_avg_std(0, 1);
		p->calculate_background();
		fft_plan planf = fft_setup_plan(p->sizeX(), p->sizeY(), 1, FFTW_FORWARD, 1);
		p->fft(planf, 0);
		fft_destroy_plan(planf);
		p->set(0, 0);
		p->set(1, 0);
		Vector3<double> scale(1,1,1);
		if ( pref->sizeX() < p->sizeX() ) {
			Vector3<long> psize(pref->sizeX(), pref->sizeY(), 1);
			scale = p->change_transform_size(psize);
		}
		p->view(View(start[i][0], start[i][1], start[i][2], start[i][3]));
		CTFparam c;
		c.volt(ctfs[i][0]);
		c.aberration_weight(0, 0, ctfs[i][1]);
		c.aberration_weight(2, 0, ctfs[i][2]);
		c.aberration_weight(2, 2, ctfs[i][3]);
		c.aberration_weight(2, -2, ctfs[i][4]);
		c.aberration_weight(4, 0, ctfs[i][5]);
		int flags = ctfs[i][6] > 0 ? APPLY_CTF : 0;
		if ( def_std > 0 ) flags |= APPLY_CTF;
		else if ( flags ) { fprintf(stderr, "refine_probe: a CTF needs def_std > 0\n"); return 4; }
		long number = 0;
		double fom = max_iter > 0 ?
			img_refine_monte(p, pref, hi_res, 0, flags, max_iter, fom_type, weight, &c, def_std,
				shift_std, view_std, max_angle, max_mag, kernel, number) :
			img_refine_grid(p, pref, hi_res, 0, flags, alpha_step, accuracy, shift_step, shift_accuracy,
				max_mag, fom_type, weight, &c, def_std, kernel, number);
		View v = p->image->view();
		Vector3<double> o = p->image->origin() / scale;
		printf("%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %ld %.17g", v[0], v[1], v[2], v[3], o[0], o[1],
			fom, p->image->FOM(), number, c.defocus_average());
		// with the magnification grid: the refined sampling of the cut transform
		if ( max_mag > 0 ) printf(" %.17g %.17g", p->image->sampling()[0], p->image->sampling()[1]);
		printf("\n");
		delete p;
	}
	return 0;
}
