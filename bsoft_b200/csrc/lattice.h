// lattice.h - the phase lattice of the gridding scatter, chosen per particle
// on the host (plain C++, no CUDA).
//
// The gridding kernel walks a particle's pixels phase by phase: the pixels
// (h0 + lh i + sh j, k0 + lk j) of one phase are gridded by the 32 lanes of
// a warp at once, each lane adding to the corners of its pixel's unit cell
// of the map with a plain shared-memory read-modify-write.  That is only
// correct if two pixels of one phase never fall in the same cell.  Two
// pixels whose pixel-step difference is (dh, dk) sit d = dh ad + dk bd apart
// in the map (ad, bd: the map displacement of one pixel step along h and k);
// they can share a cell only if |d_x|, |d_y| and |d_z| are all below 1.  So
// a lattice is safe when every nonzero lattice vector has max_c |d_c| >= 1
// (with a margin above the rounding of the per-pixel coordinates: the
// kernel forms them in FP32 relative to its tile, < 5e-6 voxel).
//
// A lattice safe for every orientation needs vectors of length >= sqrt(3)
// voxels (12 phases at half-voxel pixel steps); for one orientation the
// smallest safe lattice usually has 4 to 6 phases (the cube's section by the
// particle's plane has area 4 to 3 sqrt(3) voxels^2, and a lattice with no
// point inside a symmetric convex region needs at least a quarter of its
// area per point).  Fewer phases means fewer per-phase scans and fuller warps.
#pragma once

#include <algorithm>
#include <cmath>

namespace bsg {

struct PhaseLattice {
    int lh, lk, sh;
};

// Length (in pixel steps) beyond which a pixel-step vector cannot fail:
// sqrt(3) / (smallest singular value of [ad bd]), since max_c |d_c| >=
// |d| / sqrt(3).  Infinite when ad, bd are degenerate.
inline double lattice_reach(const double ad[3], const double bd[3], double curve = 0.0) {
    double aa = 0, ab = 0, bb = 0;
    for (int c = 0; c < 3; ++c) {
        aa += ad[c] * ad[c];
        ab += ad[c] * bd[c];
        bb += bd[c] * bd[c];
    }
    const double tr = aa + bb, det = aa * bb - ab * ab;
    const double disc = std::sqrt(std::max(0.0, tr * tr - 4.0 * det));
    const double smin2 = 0.5 * (tr - disc);
    if (!(smin2 > 0)) return HUGE_VAL;
    // a curved surface (Ewald sphere) moves two points |v| pixel steps apart
    // by at most curve |v| voxels more: |d| >= |v| (sigma_min - curve)
    const double smin = std::sqrt(smin2) - curve;
    if (!(smin > 0)) return HUGE_VAL;
    return std::sqrt(3.0) / smin * (1.0 + 1e-9) + 1e-9;
}

// True when no nonzero vector of the lattice {(lh i + sh j, lk j)} maps to a
// displacement with all three |d_c| < 1 + margin.  Only vectors shorter than
// `reach` pixel steps need checking, and of each pair +-v only one.
inline bool lattice_ok(const double ad[3], const double bd[3], int lh, int lk, int sh, double reach,
                       double curve = 0.0) {
    const double margin = 2e-5;
    const int jmax = (int)std::floor(reach / lk);
    for (int j = 0; j <= jmax; ++j) {
        const double dk = (double)lk * j;
        const int ilo = j == 0 ? 1 : (int)std::ceil((-reach - (double)sh * j) / lh);
        const int ihi = (int)std::floor((reach - (double)sh * j) / lh);
        for (int i = ilo; i <= ihi; ++i) {
            const double dh = (double)lh * i + (double)sh * j;
            if (dh * dh + dk * dk > reach * reach) continue;
            double m = 0;
            for (int c = 0; c < 3; ++c) m = std::max(m, std::fabs(dh * ad[c] + dk * bd[c]));
            if (m < 1.0 + margin + curve * std::sqrt(dh * dh + dk * dk)) return false;
        }
    }
    return true;
}

// The safe lattice with the fewest phases lh * lk (up to max_phases; fewest
// rows lk first, then the smallest shift), else the square lattice of side
// ceil(reach), which no vector shorter than `reach` belongs to; {0, 0, 0}
// when that side would not fit the 12-bit fields of pack_lattice.
// curve: bound on the extra displacement (voxels per pixel step of the
// lattice vector) of a curved insertion surface; 0 for the plane.
inline PhaseLattice choose_lattice(const double ad[3], const double bd[3], int max_phases = 16, double curve = 0.0) {
    const double reach = lattice_reach(ad, bd, curve);
    if (reach < 64.0) {
        for (int d = 1; d <= max_phases; ++d)
            for (int lk = 1; lk <= d; ++lk) {
                if (d % lk) continue;
                const int lh = d / lk;
                for (int sh = 0; sh < lh; ++sh)
                    if (lattice_ok(ad, bd, lh, lk, sh, reach, curve)) return {lh, lk, sh};
            }
    }
    if (!(reach < 4095.0)) return {0, 0, 0};
    const int L = std::max(1, (int)std::ceil(reach));
    return {L, L, 0};
}

// lh | lk << 12 | sh << 24 (0: no lattice chosen).
inline int pack_lattice(const PhaseLattice& l) {
    if (l.lh <= 0 || l.lk <= 0 || l.lh > 4095 || l.lk > 4095 || l.sh < 0 || l.sh > 127) return 0;
    return l.lh | (l.lk << 12) | (l.sh << 24);
}

}  // namespace bsg
