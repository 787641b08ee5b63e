/*
 * match_oracle.c - FP64 restatement of the reference's central-section
 * projection matching (TEST INFRASTRUCTURE ONLY; see oracle.h).
 * Filled in with the matching path.
 */
#include "oracle.h"

int orc_central_section(int N, const double* vol, const double* mat, double max_rad, double* out)
{
    (void)N; (void)vol; (void)mat; (void)max_rad; (void)out;
    return -1;
}

double orc_frc_score(int N, const double* img, const double* ref, int rmin, int rmax,
                     const double* ctf2d)
{
    (void)N; (void)img; (void)ref; (void)rmin; (void)rmax; (void)ctf2d;
    return 0.0;
}
