// Brute-force check of the gridding phase lattice (bsoft_b200/csrc/lattice.h):
// for random particle orientations, pixel steps and plane offsets, the points
// of every phase fall in distinct unit cells of the map, and no chosen
// lattice has more phases than the orientation-independent one.  Prints one
// line of statistics; exit status 1 on any failure.
#include "../bsoft_b200/csrc/lattice.h"

#include <cstdio>
#include <cstdint>
#include <random>
#include <unordered_set>

static void quat_matrix(double w, double x, double y, double z, double R[9]) {
    R[0] = w * w + x * x - y * y - z * z; R[1] = 2 * (x * y - w * z);         R[2] = 2 * (x * z + w * y);
    R[3] = 2 * (x * y + w * z);         R[4] = w * w - x * x + y * y - z * z; R[5] = 2 * (y * z - w * x);
    R[6] = 2 * (x * z - w * y);         R[7] = 2 * (y * z + w * x);         R[8] = w * w - x * x - y * y + z * z;
}

int main(int argc, char** argv) {
    const int nviews = argc > 1 ? atoi(argv[1]) : 400;
    std::mt19937_64 rng(12345);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::uniform_real_distribution<double> ud(0.0, 1.0);
    const double steps[] = {0.5, 0.4, 0.25, 0.7, 1.0};
    long hist[17] = {0};
    long checked = 0, worse = 0, collisions = 0;
    for (double step : steps) {
        for (int v = 0; v < nviews + 4; ++v) {
            double R[9];
            if (v < 4) {   // axis-aligned and diagonal views too
                const double q[4][4] = {{1, 0, 0, 0}, {0.7071067811865476, 0.7071067811865476, 0, 0},
                                        {0.8880738339771153, 0.3250575836718682, 0.3250575836718682, 0},
                                        {0.9238795325112867, 0, 0, 0.3826834323650898}};
                quat_matrix(q[v][0], q[v][1], q[v][2], q[v][3], R);
            } else {
                double w = nd(rng), x = nd(rng), y = nd(rng), z = nd(rng);
                const double n = std::sqrt(w * w + x * x + y * y + z * z);
                quat_matrix(w / n, x / n, y / n, z / n, R);
            }
            double ad[3], bd[3];
            for (int i = 0; i < 3; ++i) { ad[i] = R[3 * i + 0] * step; bd[i] = R[3 * i + 1] * step; }
            const bsg::PhaseLattice L = bsg::choose_lattice(ad, bd);
            if (L.lh <= 0) { printf("no lattice for step %g\n", step); return 1; }
            const int d = L.lh * L.lk;
            // the orientation-independent lattice the kernel used before
            const int Ls = std::max(1, (int)std::ceil(1.7320508 / step));
            const int dold = (Ls * Ls > 12 && 3.6055513 * step >= 1.7320508) ? 12 : Ls * Ls;
            if (d > dold) ++worse;
            if (step == 0.5) hist[std::min(d, 16)]++;
            const int W = 14;
            for (int off = 0; off < 6; ++off) {
                const double o[3] = {ud(rng) * 7, ud(rng) * 7, ud(rng) * 7};
                for (int pk = 0; pk < L.lk; ++pk)
                    for (int ph = 0; ph < L.lh; ++ph) {
                        std::unordered_set<int64_t> cells;
                        for (int j = -W; j <= W; ++j)
                            for (int i = -W; i <= W; ++i) {
                                const int h = ph + L.lh * i + L.sh * j, k = pk + L.lk * j;
                                int64_t key = 0;
                                for (int c = 0; c < 3; ++c) {
                                    const double m = h * ad[c] + k * bd[c] - o[c];
                                    key = key * 4096 + (int64_t)std::floor(m) + 2048;
                                }
                                if (!cells.insert(key).second) ++collisions;
                                ++checked;
                            }
                    }
            }
        }
    }
    // Ewald sphere: points on the curved surface m = h ad + k bd + kappa
    // (h^2 + k^2) n (kappa = lambda/2 inv^2 mscale, up to ~2 voxels of offset
    // at the corner of a 512^2 transform), with the lattice chosen for the
    // curvature bound kappa ft sqrt(2); windows all over the pixel square
    long curved = 0, curved_checked = 0;
    for (int v = 0; v < nviews; ++v) {
        double w = nd(rng), x = nd(rng), y = nd(rng), z = nd(rng);
        const double qn = std::sqrt(w * w + x * x + y * y + z * z);
        double R[9];
        quat_matrix(w / qn, x / qn, y / qn, z / qn, R);
        const double step = 0.5, ft = 512;
        const double kappa = (v % 3 + 1) * 1.0e-5;
        double ad[3], bd[3], nv[3];
        for (int i = 0; i < 3; ++i) { ad[i] = R[3 * i] * step; bd[i] = R[3 * i + 1] * step; nv[i] = R[3 * i + 2]; }
        const bsg::PhaseLattice L = bsg::choose_lattice(ad, bd, 16, kappa * ft * 1.4142135623730951 * 1.0001);
        if (L.lh <= 0) { printf("no curved lattice\n"); return 1; }
        const int W = 10;
        for (int win = 0; win < 4; ++win) {
            const int hc = (int)((ud(rng) * 2 - 1) * (ft / 2 - 2 * W)), kc = (int)((ud(rng) * 2 - 1) * (ft / 2 - 2 * W));
            const double o[3] = {ud(rng) * 7, ud(rng) * 7, ud(rng) * 7};
            for (int pk = 0; pk < L.lk; ++pk)
                for (int ph = 0; ph < L.lh; ++ph) {
                    std::unordered_set<int64_t> cells;
                    for (int j = -W; j <= W; ++j)
                        for (int i = -W; i <= W; ++i) {
                            const int h = hc + ph + L.lh * i + L.sh * j, k = kc + pk + L.lk * j;
                            const double ez = kappa * ((double)h * h + (double)k * k);
                            int64_t key = 0;
                            for (int c = 0; c < 3; ++c) {
                                const double m = h * ad[c] + k * bd[c] + ez * nv[c] - o[c];
                                key = key * 4096 + (int64_t)std::floor(m) + 2048;
                            }
                            if (!cells.insert(key).second) ++curved;
                            ++curved_checked;
                        }
                }
        }
    }
    // very fine steps: the square lattice of side ceil(reach) (packable), and
    // beyond the 12-bit fields no lattice at all (the kernel's own rule)
    {
        const double ad[3] = {1e-3, 0, 0}, bd[3] = {0, 1e-3, 0};
        const bsg::PhaseLattice L = bsg::choose_lattice(ad, bd);
        if (L.lh != L.lk || L.sh != 0 || L.lh < 1732 || bsg::pack_lattice(L) == 0) {
            printf("fine step: lattice %d %d %d\n", L.lh, L.lk, L.sh);
            return 1;
        }
        const double ad2[3] = {1e-4, 0, 0}, bd2[3] = {0, 1e-4, 0};
        if (bsg::pack_lattice(bsg::choose_lattice(ad2, bd2)) != 0) {
            printf("finest step: expected no lattice\n");
            return 1;
        }
    }
    printf("points %ld collisions %ld more_phases_than_before %ld phases_at_step_0.5:", checked, collisions, worse);
    for (int d = 1; d <= 16; ++d)
        if (hist[d]) printf(" %d:%ld", d, hist[d]);
    printf(" curved_points %ld curved_collisions %ld \n", curved_checked, curved);
    return (collisions || worse || curved) ? 1 : 0;
}
