// symview_probe - test harness linked against the reference library built
// from source (oracle/_ref): the view breconstruct -mode 2 picks for each
// particle, random_symmetric_view (bsoft/src/util/symmetry.cpp:816-832),
// with random() seeded by the given seed instead of getpid() (the global
// randseed flag is set, so random_seed() keeps it).  Reads "x y z angle"
// lines, prints the chosen view per line.
// Usage: symview_probe D3 12345 views.txt
#include "symmetry.h"
#include "utilities.h"
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

extern int verbose;
extern int randseed;

int main(int argc, char** argv) {
	if ( argc < 4 ) { fprintf(stderr, "usage: symview_probe sym seed views.txt\n"); return 1; }
	verbose = 0;
	Bstring s(argv[1]);
	Bsymmetry sym(s);
	srandom((unsigned) atol(argv[2]));
	randseed = 1;
	std::ifstream f(argv[3]);
	std::string line;
	while ( std::getline(f, line) ) {
		std::istringstream is(line);
		double x, y, z, a;
		if ( !(is >> x >> y >> z >> a) ) continue;
		View v(x, y, z, a);
		View r = random_symmetric_view(v, sym);
		printf("%.17g %.17g %.17g %.17g\n", r[0], r[1], r[2], r[3]);
	}
	return 0;
}
