// views_probe - test harness linked against the reference library built from
// source (oracle/_ref): prints the views of asymmetric_unit_views
// (bsoft/src/util/symmetry.cpp:383-549) for a point group, theta/phi steps in
// degrees and the flag, one "x y z angle" line per view.
// Usage: views_probe C1 3 3 1
#include "symmetry.h"
#include "utilities.h"
#include "linked_list.h"
#include <cstdio>

extern int verbose;

int main(int argc, char** argv) {
	if ( argc < 5 ) { fprintf(stderr, "usage: views_probe sym theta_deg phi_deg flag\n"); return 1; }
	verbose = 0;
	Bstring s(argv[1]);
	Bsymmetry sym(s);
	View* v = asymmetric_unit_views(sym, atof(argv[2])*M_PI/180, atof(argv[3])*M_PI/180, atoi(argv[4]));
	for ( View* w = v; w; w = w->next )
		printf("%.17g %.17g %.17g %.17g\n", (*w)[0], (*w)[1], (*w)[2], (*w)[3]);
	kill_list((char *) v, sizeof(View));
	return 0;
}
