// backproject_probe - test harness linked against the reference library built
// from source (oracle/_ref): real-space weighted back-projection of 2-D
// images into a map with the reference's own Bimage::back_project
// (bsoft/src/img/Bimage_project.cpp:466-509: ramp filter in Fourier space,
// rescale to mean 0 and standard deviation 1, trilinear sampling of the
// image along each voxel's projection), accumulated over the images as
// project_back_projection does (bsoft/src/mg/mg_reconstruct.cpp:1524-1624;
// map origin at its default, the centre).
//   in.raw   float32[K][n][n] images, x fastest
//   params   K lines "ox oy vx vy vz va" (origin in pixels, view, angle in radians)
//   out.raw  float32[N^3] map
// Usage: backproject_probe in.raw params K n pixel resolution N out.raw
#include "Bimage.h"
#include "View.h"
#include "utilities.h"

#include <cstdio>
#include <fstream>
#include <vector>

extern int verbose;

int main(int argc, char** argv) {
    if ( argc < 9 ) {
        std::cerr << "usage: backproject_probe in.raw params K n pixel resolution N out.raw" << std::endl;
        return 1;
    }
    verbose = 0;
    const long K = atol(argv[3]), n = atol(argv[4]), N = atol(argv[7]);
    const double pixel = atof(argv[5]), resolution = atof(argv[6]);
    std::vector<float> imgs(K * n * n);
    {
        std::ifstream in(argv[1], std::ios::binary);
        in.read((char*)imgs.data(), sizeof(float) * imgs.size());
        if ( !in ) return 2;
    }
    FILE* fp = fopen(argv[2], "r");
    if ( !fp ) return 2;
    Bimage* pmap = new Bimage(Float, TSimple, Vector3<long>(N, N, N), 1);
    pmap->sampling(pixel, pixel, pixel);
    pmap->origin(pmap->default_origin());
    fft_plan planf = fft_setup_plan(n, n, 1, FFTW_FORWARD, 1);
    fft_plan planb = fft_setup_plan(n, n, 1, FFTW_BACKWARD, 1);
    for ( long k = 0; k < K; ++k ) {
        double ox, oy, vx, vy, vz, va;
        if ( fscanf(fp, "%lf %lf %lf %lf %lf %lf", &ox, &oy, &vx, &vy, &vz, &va) != 6 ) return 3;
        Bimage* p = new Bimage(Float, TSimple, Vector3<long>(n, n, 1), 1);
        float* d = (float*) p->data_pointer();
        for ( long i = 0; i < n * n; ++i ) d[i] = imgs[k * n * n + i];
        p->statistics();
        p->sampling(pixel, pixel, 1);
        p->origin(Vector3<double>(ox, oy, 0));
        p->image->view(View(vx, vy, vz, va));
        p->image->magnification(1);
        pmap->back_project(p, resolution, 0, planf, planb);
        delete p;
    }
    fclose(fp);
    fft_destroy_plan(planf);
    fft_destroy_plan(planb);
    std::ofstream out(argv[8], std::ios::binary);
    out.write((const char*) pmap->data_pointer(), sizeof(float) * N * N * N);
    delete pmap;
    return 0;
}
