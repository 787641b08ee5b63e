// match_probe - test harness linked against the reference library built from
// source (oracle/_ref).  It runs the reference's own projection-matching
// steps (brefine's grid refinement: bsoft/src/mg/mg_refine.cpp:279-365 for
// the reference map, :509-563 for a particle, :862-933 for one hypothesis)
// and writes what they produce, so the oracle's restatement and the CUDA
// matching path can be pinned to it:
//   <out>.map    float[2*diam^3]          prepared reference transform
//   <out>.sec    float[2*diam^2] per view  central sections (hi_res/1.11)
//   <out>.img    float[2*diam^2] per image prepared particle transforms
//   <out>.fom    text "fom cv" per hypothesis (img_recip_space_fom; FRC, or
//                DPR with MATCH_PROBE_FOM_TYPE=1 in the environment)
// Usage:
//   match_probe map.mrc stack.mrc pixel hi_res views.txt ctf.txt hyps.txt out [width power]
// views.txt: "x y z angle(rad)" per view; ctf.txt: "volt abw00 abw20 abw22 abw2m2
// abw40 apply" per image; hyps.txt: "image view origin_x origin_y" per
// hypothesis, origins in pixels of the uncut particle image.
#include "rwimg.h"
#include "mg_processing.h"
#include "Bimage.h"
#include "FSI_Kernel.h"
#include "ctf.h"
#include "View.h"
#include "utilities.h"
#include <fstream>
#include <sstream>

extern int verbose;

// external linkage in the reference, declared in no header (mg_refine.cpp:660)
double img_recip_space_fom(Bimage* p, Bimage* pref, double hi_res, double lo_res,
                           int fom_type, vector<double>& weight, int flags, CTFparam* em_ctf);

static void append(const std::string& f, const void* p, size_t bytes, bool first) {
	std::ofstream o(f, first ? std::ios::binary : (std::ios::binary | std::ios::app));
	o.write((const char*)p, bytes);
}

int main(int argc, char** argv) {
	if ( argc < 9 ) { std::cerr << "usage: match_probe map stack pixel hi_res views ctf hyps out [w p]" << std::endl; return 1; }
	verbose = 0;
	std::string mapfile(argv[1]), stackfile(argv[2]), out(argv[8]);
	double pixel = atof(argv[3]), hi_res = atof(argv[4]);
	int kw = argc > 9 ? atoi(argv[9]) : 8, kp = argc > 10 ? atoi(argv[10]) : 2;

	// reference map: project_refine_orientations, mg_refine.cpp:279-365
	Bimage* pref = read_img(mapfile, 1, -1);
	if ( !pref ) return 2;
	pref->check_resolution(hi_res);
	Vector3<double> map_origin = pref->image->origin();
	if ( pref->compound_type() == TSimple ) pref->fft();
	int diam = (int) (2.2*pref->real_size()[0]/hi_res + 0.5);
	if ( diam%2 ) diam += 1;
	Vector3<long> size(diam, diam, diam);
	if ( diam < pref->sizeX() ) pref->change_transform_size(size);
	pref->set(0, 0);
	pref->set(1, 0);
	pref->check_resolution(hi_res);
	FSI_Kernel* kernel = new FSI_Kernel(kw, kp);
	pref->phase_shift_to_origin();
	diam = pref->sizeX();
	append(out + ".map", pref->data_pointer(), sizeof(float)*2*pref->image_size(), true);

	std::vector<View> views;
	{ std::ifstream f(argv[5]); double x, y, z, a; while ( f >> x >> y >> z >> a ) views.push_back(View(x, y, z, a)); }
	std::vector<std::vector<double>> ctfs;
	{ std::ifstream f(argv[6]); std::string line;
	  while ( std::getline(f, line) ) { std::istringstream s(line); std::vector<double> v; double t;
	    while ( s >> t ) v.push_back(t); if ( v.size() >= 7 ) ctfs.push_back(v); } }
	std::vector<std::vector<double>> hyps;
	{ std::ifstream f(argv[7]); double a, b, c, d; while ( f >> a >> b >> c >> d ) hyps.push_back({a, b, c, d}); }

	// particles: part_refine_orientation, mg_refine.cpp:509-563
	std::vector<Bimage*> imgs;
	Vector3<double> scale(1,1,1);
	for ( size_t i = 0; i < ctfs.size(); ++i ) {
		Bimage* p = read_img(stackfile, 1, (long)i);
		if ( !p ) return 3;
		p->sampling(pixel, pixel, 1);
		p->change_type(Float);
		p->rescale_to_avg_std(0, 1);
		p->calculate_background();
		fft_plan planf = fft_setup_plan(p->sizeX(), p->sizeY(), 1, FFTW_FORWARD, 1);
		p->fft(planf, 0);
		fft_destroy_plan(planf);
		p->set(0, 0);
		p->set(1, 0);
		if ( pref->sizeX() < p->sizeX() ) {
			Vector3<long> psize(pref->sizeX(), pref->sizeY(), 1);
			scale = p->change_transform_size(psize);
		}
		append(out + ".img", p->data_pointer(), sizeof(float)*2*p->image_size(), i == 0);
		imgs.push_back(p);
	}

	// sections: img_fit_in_recip_space_grid, mg_refine.cpp:868-885
	std::vector<Bimage*> secs;
	for ( size_t v = 0; v < views.size(); ++v ) {
		Bimage* p = imgs.empty() ? NULL : imgs[0];
		Vector3<double> sc = p ? pref->sampling(0)/p->sampling(0) : Vector3<double>(1,1,1);
		sc[2] = 1;
		Matrix3 mat = views[v].matrix();
		mat[0] *= sc;
		mat[1] *= sc;
		Bimage* pcs = pref->central_section(mat, hi_res/1.11, kernel);
		append(out + ".sec", pcs->data_pointer(), sizeof(float)*2*pcs->image_size(), v == 0);
		secs.push_back(pcs);
	}

	// hypotheses: mg_refine.cpp:918-924
	std::ofstream fo(out + ".fom");
	fo.precision(17);
	vector<double> weight;
	// MATCH_PROBE_FOM_TYPE=1 scores with the DPR form (brefine -fomtype dpr)
	const int fom_type = getenv("MATCH_PROBE_FOM_TYPE") ? atoi(getenv("MATCH_PROBE_FOM_TYPE")) : 0;
	for ( auto& h : hyps ) {
		long ii = (long)h[0], vv = (long)h[1];
		Bimage* pcopy = imgs[ii]->copy();
		pcopy->image->origin(Vector3<double>(h[2]*scale[0], h[3]*scale[1], 0));
		pcopy->phase_shift_to_origin();
		CTFparam c;
		c.volt(ctfs[ii][0]);
		c.aberration_weight(0, 0, ctfs[ii][1]);
		c.aberration_weight(2, 0, ctfs[ii][2]);
		c.aberration_weight(2, 2, ctfs[ii][3]);
		c.aberration_weight(2, -2, ctfs[ii][4]);
		c.aberration_weight(4, 0, ctfs[ii][5]);
		int flags = (ctfs[ii].size() > 6 && ctfs[ii][6] > 0) ? APPLY_CTF : 0;
		double fom = img_recip_space_fom(pcopy, secs[vv], hi_res, 0, fom_type, weight, flags, &c);
		fo << fom << " " << pcopy->image->FOM() << "\n";
		delete pcopy;
	}
	std::cout << "diam " << diam << " scale " << scale[0] << " map_origin " << map_origin[0] << " " << map_origin[1] << " "
		<< map_origin[2] << " hi_res " << hi_res << " map_sampling " << pref->sampling(0)[0]
		<< " img_sampling " << (imgs.empty() ? 0.0 : imgs[0]->sampling(0)[0]) << std::endl;
	return 0;
}
