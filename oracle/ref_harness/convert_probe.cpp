// convert_probe - test harness linked against the reference library built
// from source (oracle/_ref): reads an image file with read_img and writes it
// with write_img, whose output format follows the extension (e.g. .spi for
// SPIDER, bsoft/src/rwimg/rwSPIDER.cpp).  Used to make SPIDER particle stacks
// exactly as the reference writes them.
// Usage: convert_probe in.mrcs out.spi
#include "rwimg.h"
#include "utilities.h"
#include <cstdio>

extern int verbose;

int main(int argc, char** argv) {
	if ( argc < 3 ) { fprintf(stderr, "usage: convert_probe in out\n"); return 1; }
	verbose = 0;
	Bimage* p = read_img(argv[1], 1, -1);
	if ( !p ) return 2;
	if ( write_img(argv[2], p, 0) < 0 ) return 3;
	delete p;
	return 0;
}
