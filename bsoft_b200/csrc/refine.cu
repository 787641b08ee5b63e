// refine.cu - brefine's grid refinement of particle orientations and origins
// on the GPU: img_refine_grid (bsoft/src/mg/mg_refine.cpp:1086-1195) with its
// shift search img_fit_in_recip_space_grid (:862-950) and the view grid of
// views_for_refinement (bsoft/src/util/View.cpp:371-424).
//
// The reference walks one particle at a time: for each of 27 views around
// the current best (three rotations of +-alpha and 0 about two axes normal to
// the view vector, three in-plane angles), a 3 x 3 grid of origins at
// halving steps around the particle's original origin, every hypothesis
// scored by img_recip_space_fom; alpha halves when the centre view wins or
// the best figure of merit stops moving by 1e-6.
//
// Here every particle's state machine runs on the host in lockstep and each
// round scores, for every active particle, all 27 views at every shift level
// in ONE launch of the exact figure-of-merit kernel (one block per view and
// level: the section is gathered once and scored at the level's <= 9
// origins).  The shift grid is centred on the original origin at every
// level, so its levels are known before any score: the host then replays
// the reference's decisions (level repeats, best-of-level, view choice) on
// the returned scores in the reference's order, with the reference's
// floating-point loops for the view and origin grids.
#include "match.cuh"

#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

namespace bsg {
namespace {

constexpr double TRIGPREC = 1e-30;   // TRIGPRECISION / SMALLFLOAT (bsoft/include/utilities.h)
constexpr int NVIEW = 27;            // views_for_refinement: 3 x 3 x 3
constexpr int MAX_LEVELS = 32;       // shift grid levels (shift_step / shift_accuracy <= 2^31)
constexpr long MAX_ROUNDS = 100000;  // angular rounds per particle (the reference has no bound)

// angle_set_negPI_to_PI (bsoft/src/util/utilities.cpp:606-615)
double angle_neg_pi_to_pi(double a) {
    if (!isfinite(a)) return 0;
    const long n = (long)(a / M_PI);
    a -= (n + n % 2) * M_PI;
    return a;
}

struct Vec3 {
    double d[3];
    double length2() const { return d[0] * d[0] + d[1] * d[1] + d[2] * d[2]; }
    double length() const { return sqrt(length2()); }
    // Vector3::normalize (bsoft/include/Vector3.h:264-274)
    void normalize() {
        const double len = length();
        if (len < 1e-30) {
            d[2] = 1;
        } else {
            const double div = 1.0 / len;
            for (int i = 0; i < 3; ++i) d[i] *= div;
        }
    }
    Vec3 cross(const Vec3& v) const {
        return Vec3{{d[1] * v.d[2] - d[2] * v.d[1], d[2] * v.d[0] - d[0] * v.d[2], d[0] * v.d[1] - d[1] * v.d[0]}};
    }
};

// View: unit view vector and in-plane angle (bsoft/include/View.h); every
// construction and copy of a View in the reference renormalises it
// (View.h:40-52, normalize/check :30-35, 110-116)
struct View4 {
    double v[3], a;
    void normalize() {
        const double size = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (size < TRIGPREC) {
            v[0] = v[1] = 0;
            v[2] = 1;
        } else {
            v[0] /= size;
            v[1] /= size;
            v[2] /= size;
        }
        for (int i = 0; i < 3; ++i)
            if (fabs(v[i]) < TRIGPREC) v[i] = 0;
        a = angle_neg_pi_to_pi(a);
        if (fabs(a) < TRIGPREC) a = 0;
    }
};

View4 make_view(double x, double y, double z, double a) {
    View4 w{{x, y, z}, a};
    w.normalize();
    return w;
}

View4 renormalised(View4 w, int times) {
    for (int t = 0; t < times; ++t) w.normalize();
    return w;
}

// Quaternion (bsoft/include/Quaternion.h): scalar s, vector v
struct Quat {
    double s, v[3];
    void check() {
        if (fabs(s) < TRIGPREC) s = 0;
        for (int i = 0; i < 3; ++i)
            if (fabs(v[i]) < TRIGPREC) v[i] = 0;
    }
    // from_axis_angle (Quaternion.h:34-41)
    static Quat axis_angle(const Vec3& axis, double angle) {
        const double a = angle / 2.0;
        Vec3 u = axis;
        u.normalize();
        Quat q{cos(a), {0, 0, 0}};
        const double sa = sin(a);
        for (int i = 0; i < 3; ++i) q.v[i] = u.d[i] * sa;
        q.check();
        return q;
    }
    // Hamilton product (Quaternion.h:117-124)
    Quat operator*(const Quat& q) const {
        Quat n;
        n.s = s * q.s - (v[0] * q.v[0] + v[1] * q.v[1] + v[2] * q.v[2]);
        n.v[0] = s * q.v[0] + v[0] * q.s + v[1] * q.v[2] - v[2] * q.v[1];
        n.v[1] = s * q.v[1] + v[1] * q.s + v[2] * q.v[0] - v[0] * q.v[2];
        n.v[2] = s * q.v[2] + v[2] * q.s + v[0] * q.v[1] - v[1] * q.v[0];
        return n;
    }
    // rotate(point) = q point q^-1, the inverse by invert() (Quaternion.h:161-177)
    Quat rotate(const Quat& p) const {
        Quat inv = *this;
        inv.check();
        const double size2 = inv.s * inv.s + (inv.v[0] * inv.v[0] + inv.v[1] * inv.v[1] + inv.v[2] * inv.v[2]);
        const double div = 1 / size2;
        inv.s *= div;
        for (int i = 0; i < 3; ++i) inv.v[i] *= -div;
        return (*this * p) * inv;
    }
};

// View::quaternion then Matrix3(Quaternion) (View.h:131-157, Matrix3.h:21-42)
void view_matrix(View4 w, double* m) {
    w.normalize();
    const double ang = w.a / 2.0;
    const double ca = cos(ang), sa = sin(ang);
    const double z1 = w.v[2] + 1;
    double q[4] = {ca, 0, 0, sa};
    if (w.v[2] < 1.0 - TRIGPREC) {
        if (w.v[2] <= TRIGPREC - 1.0) {
            q[0] = 0;
            q[1] = sa;
            q[2] = ca;
            q[3] = 0;
        } else {
            const double f1 = sqrt(z1 / 2.0), f2 = sqrt(1.0 / (2 * z1));
            q[0] = f1 * ca;
            q[1] = f2 * (w.v[0] * sa - w.v[1] * ca);
            q[2] = f2 * (w.v[0] * ca + w.v[1] * sa);
            q[3] = f1 * sa;
        }
    }
    for (int i = 0; i < 4; ++i)
        if (fabs(q[i]) < TRIGPREC) q[i] = 0;
    m[0] = q[0] * q[0] + q[1] * q[1] - q[2] * q[2] - q[3] * q[3];
    m[1] = 2 * q[1] * q[2] - 2 * q[0] * q[3];
    m[2] = 2 * q[1] * q[3] + 2 * q[0] * q[2];
    m[3] = 2 * q[1] * q[2] + 2 * q[0] * q[3];
    m[4] = q[0] * q[0] - q[1] * q[1] + q[2] * q[2] - q[3] * q[3];
    m[5] = 2 * q[2] * q[3] - 2 * q[0] * q[1];
    m[6] = 2 * q[1] * q[3] - 2 * q[0] * q[2];
    m[7] = 2 * q[2] * q[3] + 2 * q[0] * q[1];
    m[8] = q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3];
    for (int i = 0; i < 9; ++i) {
        if (fabs(m[i]) < 1e-12) m[i] = 0;
        if (m[i] > 1) m[i] = 1;
        if (m[i] < -1) m[i] = -1;
    }
}

// views_for_refinement (View.cpp:371-424): theview is the by-value copy
// (one renormalisation) that the function normalises once more
int views_for_refinement(View4 theview, double alpha_step, View4* out) {
    int nv = 0;
    if (alpha_step <= 0) {
        out[nv++] = theview;
        return nv;
    }
    theview.normalize();
    const Vec3 ref_axis{{0, 0, 1}};
    const Vec3 vv{{theview.v[0], theview.v[1], theview.v[2]}};
    Vec3 axis1 = vv.cross(ref_axis);
    if (axis1.length() < 0.001) axis1.d[0] = 1;
    axis1.normalize();
    Vec3 axis2 = vv.cross(axis1);
    if (axis2.length() < 0.001) axis2.d[1] = 1;
    axis2.normalize();
    Quat qv{0, {theview.v[0], theview.v[1], theview.v[2]}};
    qv.check();
    for (double alpha1 = -alpha_step; alpha1 <= alpha_step; alpha1 += alpha_step) {
        const Quat q1 = Quat::axis_angle(axis1, alpha1);
        for (double alpha2 = -alpha_step; alpha2 <= alpha_step; alpha2 += alpha_step) {
            Quat q = Quat::axis_angle(axis2, alpha2);
            q = q * q1;
            q = q.rotate(qv);
            for (double alpha3 = -alpha_step; alpha3 <= alpha_step; alpha3 += alpha_step) {
                if (nv < NVIEW) out[nv] = make_view(q.v[0], q.v[1], q.v[2], theview.a + alpha3);
                ++nv;
            }
        }
    }
    return nv;
}

// One level of the origin grid (img_fit_in_recip_space_grid :917-919): the
// reference's floating loops from o - step to o + step, y outer, x inner
struct Level {
    double x[MAXORG], y[MAXORG];
    int n;
};

Level origin_level(double ox, double oy, double step) {
    Level L;
    L.n = 0;
    for (double y = oy - step; y <= oy + step; y += step)
        for (double x = ox - step; x <= ox + step; x += step) {
            if (L.n < MAXORG) {
                L.x[L.n] = x;
                L.y[L.n] = y;
            }
            ++L.n;
        }
    return L;
}

struct Particle {
    long img;
    double ox, oy;                 // original origin, pixels of the cut transform
    std::vector<Level> levels;     // shift grid levels, largest step first
    View4 bestview;
    double alpha, prefom, bestfom, bestcv, box, boy;
    long number;
    long rounds;
    bool done;
    View4 views[NVIEW];            // this round's views
};

}  // namespace
}  // namespace bsg

using namespace bsg;

extern "C" int bsg_match_refine(bsg_match* h, const double* start, long nstart, double alpha_step, double accuracy,
                                double shift_step, double shift_accuracy, double* out, int flags) {
    (void)flags;
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !start || !out || nstart < 1) return match_fail(BSG_ERR_ARG, "bsg_match_refine: bad argument");
    if (!M->have_ref || M->nimg < 1)
        return match_fail(BSG_ERR_STATE, "bsg_match_refine: set the reference and images first");
    // img_refine_grid's own checks (mg_refine.cpp:1091-1103)
    if (!(alpha_step >= TRIGPREC) || !(accuracy >= TRIGPREC))
        return match_fail(BSG_ERR_ARG, "bsg_match_refine: angular step %g or accuracy %g too small", alpha_step,
                          accuracy);
    if (alpha_step < accuracy)
        return match_fail(BSG_ERR_ARG, "bsg_match_refine: angular step %g smaller than the accuracy %g", alpha_step,
                          accuracy);
    // the reference's shift loop never ends for a non-positive accuracy
    if (!(shift_accuracy > 0) || !isfinite(shift_step))
        return match_fail(BSG_ERR_ARG, "bsg_match_refine: shift accuracy must be positive (got %g)", shift_accuracy);
    std::vector<double> steps;
    for (double st = shift_step; st >= shift_accuracy; st /= 2) {
        if ((int)steps.size() >= MAX_LEVELS)
            return match_fail(BSG_ERR_ARG, "bsg_match_refine: more than %d shift levels (step %g, accuracy %g)",
                              MAX_LEVELS, shift_step, shift_accuracy);
        steps.push_back(st);
    }
    const int nlev = (int)steps.size();
    cudaError_t ce = cudaSetDevice(M->device);
    if (ce != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_refine: %s", cudaGetErrorString(ce));

    std::vector<Particle> parts(nstart);
    for (long i = 0; i < nstart; ++i) {
        const double* r = start + BSG_MATCH_REFINE_START_DOUBLES * i;
        const long img = (long)r[0];
        if (!(r[0] >= 0) || img >= M->nimg)
            return match_fail(BSG_ERR_ARG, "bsg_match_refine: start record %ld names image %g", i, r[0]);
        Particle& P = parts[i];
        P.img = img;
        // origin in pixels of the uncut image, scaled with the transform cut
        // (Bimage_fft.cpp:433)
        P.ox = M->cut_scale * r[5];
        P.oy = M->cut_scale * r[6];
        for (int k = 0; k < nlev; ++k) {
            P.levels.push_back(origin_level(P.ox, P.oy, steps[k]));
            if (P.levels.back().n > MAXORG)
                return match_fail(BSG_ERR_ARG, "bsg_match_refine: origin grid of %d points", P.levels.back().n);
        }
        // the particle's view as img_refine_grid holds it: constructed, stored
        // through Bimage::view, read back and copied into bestview
        P.bestview = renormalised(make_view(r[1], r[2], r[3], r[4]), 3);
        P.alpha = alpha_step;
        P.prefom = -1;
        P.bestfom = -1;
        P.bestcv = 0;
        P.box = P.ox;
        P.boy = P.oy;
        P.number = 0;
        P.rounds = 0;
        P.done = nlev == 0;    // nothing is scored: the start pose is returned
    }

    // rounds: every active particle's 27 views x nlev levels in one launch;
    // particles are taken in chunks so that a launch holds at most ~64k groups
    const long per_part = (long)NVIEW * nlev;
    const long chunk = std::max(1L, (long)(65536 / std::max(1L, per_part)));
    cudaStream_t s = M->stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float tsum = 0;
    long launches = 0;
    std::vector<MHypG> groups;
    std::vector<long> owner;
    std::vector<double> go;
    int rc = BSG_OK;
    for (long c0 = 0; c0 < nstart && rc == BSG_OK; c0 += chunk) {
        const long c1 = std::min(nstart, c0 + chunk);
        for (;;) {
            groups.clear();
            owner.clear();
            for (long i = c0; i < c1; ++i) {
                Particle& P = parts[i];
                if (P.done) continue;
                const int nv = views_for_refinement(renormalised(P.bestview, 1), P.alpha, P.views);
                if (nv != NVIEW) {
                    rc = match_fail(BSG_ERR_STATE, "bsg_match_refine: %d refinement views", nv);
                    break;
                }
                for (int v = 0; v < NVIEW; ++v) {
                    // Bimage::view stores a twice-copied view; the fit reads it
                    // back (one more) and View::matrix normalises once more
                    double mat[9];
                    view_matrix(renormalised(P.views[v], 3), mat);
                    MHypG g;
                    memset(&g, 0, sizeof(g));
                    match_view_rows(*M, mat, g.m);
                    g.img = (int)P.img;
                    for (int k = 0; k < nlev; ++k) {
                        const Level& L = P.levels[k];
                        g.norg = L.n;
                        for (int o = 0; o < L.n; ++o) {
                            // phase_shift_to_origin's slopes, as bsg_match_score
                            g.sx[o] = L.x[o] / M->D * 2 * M_PI;
                            g.sy[o] = L.y[o] / M->D * 2 * M_PI;
                        }
                        groups.push_back(g);
                    }
                }
                owner.push_back(i);
            }
            if (rc != BSG_OK || owner.empty()) break;
            const long ng = (long)groups.size();
            rc = ensure_groups(*M, ng);
            if (rc != BSG_OK) break;
            go.resize(2 * ng * MAXORG);
            ce = cudaMemcpyAsync(M->d_grp, groups.data(), sizeof(MHypG) * ng, cudaMemcpyHostToDevice, s);
            if (ce == cudaSuccess) ce = cudaEventRecord(e0, s);
            if (ce == cudaSuccess) ce = launch_fom(*M, M->d_grp, ng, M->d_gout, M->d_gout + ng * MAXORG, s, true);
            if (ce == cudaSuccess) ce = cudaEventRecord(e1, s);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(go.data(), M->d_gout, sizeof(double) * go.size(), cudaMemcpyDeviceToHost, s);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
            if (ce != cudaSuccess) {
                rc = match_fail(BSG_ERR_CUDA, "bsg_match_refine: %s", cudaGetErrorString(ce));
                break;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            tsum += ms;
            ++launches;
            const double* gfom = go.data();
            const double* gcv = go.data() + ng * MAXORG;
            for (size_t t = 0; t < owner.size(); ++t) {
                Particle& P = parts[owner[t]];
                const long gbase = (long)t * per_part;
                // img_refine_grid's angular round (mg_refine.cpp:1112-1136)
                P.prefom = P.bestfom;
                P.bestfom = -1;
                int ibest = 0;
                for (int v = 0; v < NVIEW; ++v) {
                    // img_fit_in_recip_space_grid's shift levels (:914-944)
                    double bestfom = -1, prevfom, bestcv = 0, bx = P.ox, by = P.oy;
                    int k = 0;
                    while (k < nlev) {
                        const Level& L = P.levels[k];
                        const long g = gbase + (long)v * nlev + k;
                        prevfom = bestfom;
                        bestfom = -1;
                        int ib = 0;
                        for (int o = 0; o < L.n; ++o) {
                            const double f = gfom[g * MAXORG + o];
                            P.number++;
                            if (bestfom < f) {
                                bestfom = f;
                                ib = o;
                                bx = L.x[o];
                                by = L.y[o];
                                bestcv = gcv[g * MAXORG + o];
                            }
                        }
                        if (ib == L.n / 2 || fabs(prevfom - bestfom) < 1e-6) ++k;
                    }
                    if (P.bestfom < bestfom) {
                        P.bestfom = bestfom;
                        ibest = v;
                        P.bestview = P.views[v];
                        P.box = bx;
                        P.boy = by;
                        P.bestcv = bestcv;
                    }
                }
                if (ibest == NVIEW / 2 || fabs(P.prefom - P.bestfom) < 1e-6) P.alpha /= 2;
                if (!(P.alpha >= accuracy) || ++P.rounds >= MAX_ROUNDS) P.done = true;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != BSG_OK) return rc;
    for (long i = 0; i < nstart; ++i) {
        const Particle& P = parts[i];
        // p->view(bestview) stores a twice-copied view; reading it back copies once more
        const View4 w = renormalised(P.bestview, 3);
        double* o = out + BSG_MATCH_REFINE_RESULT_DOUBLES * i;
        o[0] = w.v[0];
        o[1] = w.v[1];
        o[2] = w.v[2];
        o[3] = w.a;
        o[4] = P.box / M->cut_scale;
        o[5] = P.boy / M->cut_scale;
        o[6] = P.bestfom;
        o[7] = P.bestcv;
        o[8] = (double)P.number;
    }
    M->sstats.refine_ms += tsum;
    M->sstats.refine_launches += launches;
    M->sstats.launches += launches;
    return BSG_OK;
}
