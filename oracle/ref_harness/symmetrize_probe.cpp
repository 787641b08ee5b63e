// symmetrize_probe - test harness linked against the reference library built
// from source (oracle/_ref): applies the reference's real-space point-group
// symmetrization, Bimage::symmetrize(Bsymmetry, 1) (bsoft/src/img/
// Bimage_symmetry.cpp:31-100, breconstruct's -symmetry with sym_mode 1,
// breconstruct.cpp:335), to a raw float map and writes the result.
//   in.raw / out.raw   float32[N^3], x fastest
// Prints the symmetry FOM and the background the reference used as the fill.
// With symmetry "rot:ax,ay,az,angle" it writes one Bimage::rotate instead.
// Usage: symmetrize_probe in.raw N ox oy oz symmetry out.raw
#include "Bimage.h"
#include "symmetry.h"

#include <cstdio>
#include <fstream>
#include <vector>

extern int verbose;

int main(int argc, char** argv) {
    if ( argc < 8 ) { std::cerr << "usage: symmetrize_probe in.raw N ox oy oz symmetry out.raw" << std::endl; return 1; }
    verbose = 0;
    const long N = atol(argv[2]);
    std::vector<float> buf(N * N * N);
    {
        std::ifstream in(argv[1], std::ios::binary);
        in.read((char*)buf.data(), sizeof(float) * buf.size());
        if ( !in ) return 2;
    }
    Bimage* p = new Bimage(Float, TSimple, Vector3<long>(N, N, N), 1);
    float* d = (float*) p->data_pointer();
    for ( size_t i = 0; i < buf.size(); ++i ) d[i] = buf[i];
    p->statistics();
    p->origin(Vector3<double>(atof(argv[3]), atof(argv[4]), atof(argv[5])));
    Bstring label(argv[6]);
    if ( label.length() > 4 && label.substr(0, 4) == "rot:" ) {
        // one rotation, Bimage::rotate(size, axis, angle): rot:ax,ay,az,angle
        double ax, ay, az, ang;
        if ( sscanf(argv[6] + 4, "%lf,%lf,%lf,%lf", &ax, &ay, &az, &ang) != 4 ) return 3;
        p->calculate_background();
        Bimage* pr = p->rotate(p->size(), Vector3<double>(ax, ay, az), ang);
        std::ofstream out(argv[7], std::ios::binary);
        out.write((const char*) pr->data_pointer(), sizeof(float) * N * N * N);
        printf("background %.17g rotated_background %.17g\n", p->background(long(0)), pr->background(long(0)));
        delete pr;
        delete p;
        return 0;
    }
    Bsymmetry sym(label);
    if ( getenv("SYMMETRIZE_PROBE_OPS") )
        for ( long i = 0; i < sym.operations(); ++i )
            fprintf(stderr, "op %ld axis %.17g %.17g %.17g order %d\n", i, sym[i].axis()[0], sym[i].axis()[1],
                    sym[i].axis()[2], sym[i].order());
    p->calculate_background();
    const double bkg0 = p->background(long(0));
    const double f = p->symmetrize(sym, 1);
    d = (float*) p->data_pointer();
    std::ofstream out(argv[7], std::ios::binary);
    out.write((const char*)d, sizeof(float) * N * N * N);
    printf("order %ld fom %.9g background_before %.9g background_after %.9g\n", (long) sym.order(), f, bkg0,
           p->background(long(0)));
    delete p;
    return 0;
}
