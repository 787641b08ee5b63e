// fsc_probe - test harness linked against the reference library built from
// source (oracle/_ref): the Fourier shell correlation of two maps as
// bresolve computes it for complex input (bsoft/src/bresolve.cpp:165-169):
// both maps transformed with Bimage::fft(), then Bimage::fsc(Bimage*)
// (bsoft/src/img/Bimage_resolution.cpp:330-406).  Prints one FSC value per
// shell.
// Usage: fsc_probe map1.mrc map2.mrc hi_res
#include "rwimg.h"
#include "Bimage.h"
#include "Bplot.h"
#include "utilities.h"
#include <cstdio>

extern int verbose;

int main(int argc, char** argv) {
	if ( argc < 4 ) { fprintf(stderr, "usage: fsc_probe map1 map2 hi_res\n"); return 1; }
	verbose = 0;
	Bimage* p = read_img(argv[1], 1, -1);
	Bimage* pr = read_img(argv[2], 1, -1);
	if ( !p || !pr ) return 2;
	p->fft();
	pr->fft();
	Bplot* plot = p->fsc(pr, atof(argv[3]), 1);
	for ( long i = 0; i < plot->rows(); ++i ) printf("%.17g %.17g\n", (*plot)[i], (*plot)[plot->rows() + i]);
	return 0;
}
