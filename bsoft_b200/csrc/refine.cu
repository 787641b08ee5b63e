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
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

namespace bsg {
namespace {

constexpr double TRIGPREC = 1e-30;   // TRIGPRECISION / SMALLFLOAT (bsoft/include/utilities.h)
constexpr int NVIEW = 27;            // views_for_refinement: 3 x 3 x 3
constexpr int MAX_LEVELS = 32;       // shift grid levels (shift_step / shift_accuracy <= 2^31)
constexpr long MAX_ROUNDS = 100000;  // angular rounds per particle (the reference has no bound)
constexpr int MAX_MAG_STEPS = 64;    // magnification factors per axis (the reference's grid has 21)

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

// CTFparam's defocus accessors (bsoft/include/ctf.h:133-134): abw[2,0] =
// t2 * defocus with the wavelength term t2 = -pi lambda held as a long
// double (ctf.h:48, 76-79) and lambda from ctf.h:309-317 (constants of
// bsoft/include/utilities.h:55-58).  The defocus search's floating loop
// visits def - 5 sigma .. def + 5 sigma; whether its last step is taken
// depends on the last bit of def, so the long double rounding is kept.
struct DefocusTerm {
    long double t2 = 0;
    explicit DefocusTerm(double volt) {
        const double planck = 6.626070E-34, emass = 9.109384E-31, echarge = 1.602177E-19, light = 299792458;
        const double root = sqrt(2.0 * emass * echarge * volt * (1.0 + echarge * volt / (2.0 * emass * light * light)));
        const double wl = (double)((long double)planck * 1e10L / (long double)root);
        t2 = (long double)(-M_PI * wl);
    }
    double abw20(double defocus) const { return (double)(t2 * (long double)defocus); }
    double defocus(double abw20) const { return (double)((long double)abw20 / t2); }
};

constexpr int MAX_DEF = 64;          // defocus trials per view (the reference's loop makes 10 or 11)

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
    // defocus search (brefine -defocus)
    double def0 = 0;               // img_refine_grid's `def`: the particle's defocus
    double bestdef = 0;
    std::vector<double> dvals;     // the fit's defocus trials; row dvals.size() = no trial won
    long row0 = 0;                 // first row of this particle in the call's CTF table
    int vk[NVIEW];                 // this round: chosen trial per view
    double vfom[NVIEW], vcv[NVIEW];
    double bmx = 1, bmy = 1;       // magnification stage: the winning per-axis sampling factors
};

}  // namespace
}  // namespace bsg

using namespace bsg;

extern "C" int bsg_match_refine(bsg_match* h, const double* start, long nstart, double alpha_step, double accuracy,
                                double shift_step, double shift_accuracy, double def_std, double max_mag, double* out,
                                int flags) {
    const bool dpr = (flags & BSG_MATCH_SCORE_DPR) != 0;
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
    if (!(def_std >= 0) || !isfinite(def_std))
        return match_fail(BSG_ERR_ARG, "bsg_match_refine: bad defocus step %g", def_std);
    // img_refine_grid's magnification grid (mg_refine.cpp:1151-1154): factors
    // 1 - max_mag .. 1 + max_mag in floating steps of max_mag / 10, y outer
    std::vector<std::pair<double, double>> mags;
    if (!(max_mag >= 0) || !(max_mag < 1))
        return match_fail(BSG_ERR_ARG, "bsg_match_refine: magnification range %g outside [0, 1)", max_mag);
    if (max_mag > 0) {
        const double mmin = 1.0 - max_mag, mmax = 1.0 + max_mag, mstep = max_mag / 10;
        std::vector<double> axis;
        for (double m = mmin; m <= mmax; m += mstep) {
            if ((int)axis.size() >= MAX_MAG_STEPS || m + mstep == m)
                return match_fail(BSG_ERR_ARG, "bsg_match_refine: magnification step %g too small", mstep);
            axis.push_back(m);
        }
        for (double my : axis)
            for (double mx : axis) mags.push_back({mx, my});
    }
    std::vector<double> steps;
    for (double st = shift_step; st >= shift_accuracy; st /= 2) {
        if ((int)steps.size() >= MAX_LEVELS)
            return match_fail(BSG_ERR_ARG, "bsg_match_refine: more than %d shift levels (step %g, accuracy %g)",
                              MAX_LEVELS, shift_step, shift_accuracy);
        steps.push_back(st);
    }
    const int nlev = (int)steps.size();
    const bool dsearch = def_std > 0;
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
        P.done = nlev == 0 && !dsearch;    // nothing is scored: the start pose is returned
        if (dsearch) {
            // img_refine_grid :1105-1106, the view loop's reset :1118 and the
            // fit's defocus trials :866-871, 892, 899
            const double volt = M->h_volt[img];
            if (!(volt > 0))
                return match_fail(BSG_ERR_ARG, "bsg_match_refine: image %ld has no voltage for the defocus search", img);
            const DefocusTerm dz(volt);
            P.def0 = P.bestdef = dz.defocus(M->h_ictf[img].c[1]);
            if (P.def0 == 0)
                return match_fail(BSG_ERR_ARG, "bsg_match_refine: image %ld has no defocus to search around", img);
            const double b = dz.defocus(dz.abw20(P.def0));
            const double d0 = b - 5 * def_std, d1 = b + 5 * def_std;
            for (double d = d0; d <= d1; d += def_std) {
                if ((int)P.dvals.size() >= MAX_DEF || d + def_std == d)
                    return match_fail(BSG_ERR_ARG, "bsg_match_refine: defocus step %g too small for defocus %g",
                                      def_std, P.def0);
                P.dvals.push_back(d);
            }
            P.dvals.push_back(b);    // the row used when no trial improves on -1
        }
    }

    // rounds: every active particle's 27 views gathered once (FP64 section
    // values at the figure-of-merit pixels), then scored in one launch per
    // pass (defocus trials, then shift levels); particles are taken in chunks
    // so that a launch holds at most ~64k groups and the gathered sections
    // at most ~1 GB
    const int npix = (int)M->h_pix.size();
    const long per_b = (long)NVIEW * std::max(nlev, 1);
    const long per_a = dsearch ? (long)NVIEW * (MAX_DEF / 4) : 0;
    const long sec_views = std::max((long)NVIEW, (long)((1L << 30) / ((long)sizeof(double2) * std::max(npix, 1))));
    const long chunk = std::max(1L, std::min((long)(65536 / std::max(per_a, per_b)), sec_views / NVIEW));
    cudaStream_t s = M->stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float tsum = 0;
    long launches = 0;
    std::vector<MHypG> groups;
    std::vector<long> owner, gfirst;
    std::vector<double> go;
    float* d_rctf = nullptr;
    ImgCtf* d_rrec = nullptr;
    double* d_rmats = nullptr;          // chunk x 27 views, 9 doubles each
    double2* d_sec = nullptr;           // chunk x 27 gathered sections
    std::vector<double> mats;
    int rc = BSG_OK;
    {
        const long nvmax = std::min(nstart, chunk) * NVIEW;
        ce = cudaMalloc(&d_rmats, sizeof(double) * 9 * nvmax);
        if (ce == cudaSuccess) ce = cudaMalloc(&d_sec, sizeof(double2) * (size_t)npix * nvmax);
        if (ce != cudaSuccess) {
            cudaFree(d_rmats);
            cudaFree(d_sec);
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return match_fail(BSG_ERR_NOMEM, "bsg_match_refine: %s", cudaGetErrorString(ce));
        }
    }

    // score `groups` (FP64) with the given CTF table and gathered sections;
    // results in go
    auto score_with = [&](const float* table, const double2* sec) -> int {
        const long ng = (long)groups.size();
        int r = ensure_groups(*M, ng);
        if (r != BSG_OK) return r;
        go.resize(2 * ng * MAXORG);
        cudaError_t e = cudaMemcpyAsync(M->d_grp, groups.data(), sizeof(MHypG) * ng, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaEventRecord(e0, s);
        if (e == cudaSuccess)
            e = launch_fom(*M, M->d_grp, ng, M->d_gout, M->d_gout + ng * MAXORG, s, true, table, sec, dpr);
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(go.data(), M->d_gout, sizeof(double) * go.size(), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_refine: %s", cudaGetErrorString(e));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        tsum += ms;
        ++launches;
        return BSG_OK;
    };
    auto score = [&](const float* table) -> int { return score_with(table, d_sec); };
    // group of the t-th active particle's view v (its gathered section t * 27 + v)
    auto view_group = [&](const Particle& P, long t, int v) {
        MHypG g;
        memset(&g, 0, sizeof(g));
        memcpy(g.m, &mats[9 * (t * NVIEW + v)], sizeof(g.m));
        g.img = (int)P.img;
        g.ctf = (int)P.img;
        g.sec = (int)(t * NVIEW + v);
        return g;
    };
    // phase_shift_to_origin's slopes, as bsg_match_score forms them
    auto slope = [&](double o) { return o / M->D * 2 * M_PI; };

    // img_refine_grid's magnification stage (mg_refine.cpp:1145-1187), after
    // the angular rounds: for every factor pair (mx, my), in grid order, the
    // particle's sampling becomes (s mx, s my); the best view's section is
    // gathered with rows 0 and 1 scaled by (pref sampling / that sampling) per
    // axis (img_fit_in_recip_space_grid :873-882), the CTF uses the per-axis
    // frequency steps 1 / (D s mx), 1 / (D s my) (img_recip_space_fom :694),
    // and the fit runs its defocus trials (with -defocus, around the
    // particle's defocus) and shift levels 0.4, 0.2, 0.1 around the best
    // origin of the angular stage.  A fit replaces the best one only when it
    // scores strictly higher; the best fom restarts at -1.
    const double mag_samp = M->cfg.pixel / M->cut_scale;    // Bimage::change_transform_size's sampling
    const double ref_samp = M->cfg.map_sampling / (double)((long double)M->D / M->N);
    std::vector<double> mag_steps;
    for (double st = 0.4; st >= 0.1; st /= 2) mag_steps.push_back(st);
    auto mag_stage = [&](long c0, long c1) -> int {
        const long nmag = (long)mags.size();
        long maxd = 1;
        for (long i = c0; i < c1; ++i) maxd = std::max(maxd, (long)parts[i].dvals.size());
        const long per_sec = nmag * (long)npix * (long)sizeof(double2);
        const long per_ctf = nmag * maxd * (long)npix * (long)sizeof(float);
        long sub = std::max(1L, (1L << 30) / std::max(per_sec, 1L));
        sub = std::min(sub, std::max(1L, (1L << 30) / std::max(per_ctf, 1L)));
        sub = std::min(sub, std::max(1L, 65536L / (nmag * std::max(maxd, 3L))));
        sub = std::min(sub, c1 - c0);
        double* d_mm = nullptr;
        double2* d_msec = nullptr;
        float* d_mctf = nullptr;
        ImgCtf* d_mrec = nullptr;
        cudaError_t e = cudaMalloc(&d_mm, sizeof(double) * 9 * sub * nmag);
        if (e == cudaSuccess) e = cudaMalloc(&d_msec, sizeof(double2) * (size_t)npix * sub * nmag);
        if (e == cudaSuccess) e = cudaMalloc(&d_mctf, sizeof(float) * (size_t)npix * sub * nmag * maxd);
        if (e == cudaSuccess) e = cudaMalloc(&d_mrec, sizeof(ImgCtf) * sub * nmag * maxd);
        int r = BSG_OK;
        if (e != cudaSuccess) r = match_fail(BSG_ERR_NOMEM, "bsg_match_refine: magnification stage: %s", cudaGetErrorString(e));
        std::vector<double> mm;
        std::vector<ImgCtf> recs;
        for (long p0 = c0; p0 < c1 && r == BSG_OK; p0 += sub) {
            const long p1 = std::min(c1, p0 + sub), np_ = p1 - p0;
            std::vector<std::vector<Level>> lev(np_);
            for (long t = 0; t < np_; ++t) {
                const Particle& P = parts[p0 + t];
                for (double st : mag_steps) {
                    lev[t].push_back(origin_level(P.box, P.boy, st));
                    if (lev[t].back().n > MAXORG) {
                        r = match_fail(BSG_ERR_ARG, "bsg_match_refine: origin grid of %d points", lev[t].back().n);
                        break;
                    }
                }
            }
            if (r != BSG_OK) break;
            // sections of the best views, one per factor pair
            mm.assign(9 * np_ * nmag, 0.0);
            for (long t = 0; t < np_; ++t) {
                double mat[9];
                view_matrix(renormalised(parts[p0 + t].bestview, 3), mat);
                for (long m = 0; m < nmag; ++m) {
                    const double kx = ref_samp / (mag_samp * mags[m].first);
                    const double ky = ref_samp / (mag_samp * mags[m].second);
                    double* o = &mm[9 * (t * nmag + m)];
                    for (int a = 0; a < 3; ++a)
                        for (int c = 0; c < 3; ++c) {
                            double v = mat[3 * a + c];
                            if (a < 2) v *= (c == 0 ? kx : (c == 1 ? ky : 1.0));
                            o[3 * a + c] = v;
                        }
                }
            }
            e = cudaMemcpyAsync(d_mm, mm.data(), sizeof(double) * mm.size(), cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaEventRecord(e0, s);
            if (e == cudaSuccess) e = launch_secgather(*M, d_mm, np_ * nmag, d_msec, s);
            if (e == cudaSuccess) e = cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) { r = match_fail(BSG_ERR_CUDA, "bsg_match_refine: %s", cudaGetErrorString(e)); break; }
            {
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                tsum += ms;
                ++launches;
            }
            // CTF rows at the factor pairs' frequency steps: every defocus
            // trial with -defocus, else the image's own record
            bool need_rows = dsearch;
            for (long t = 0; t < np_; ++t) need_rows = need_rows || M->h_ictf[parts[p0 + t].img].apply;
            std::vector<long> rowbase(np_, 0), nd(np_, 1);
            recs.clear();
            if (need_rows) {
                for (long t = 0; t < np_; ++t) {
                    const Particle& P = parts[p0 + t];
                    rowbase[t] = (long)recs.size();
                    nd[t] = dsearch ? (long)P.dvals.size() : 1;
                    const DefocusTerm dz(dsearch ? M->h_volt[P.img] : 0.0);
                    for (long m = 0; m < nmag; ++m) {
                        const double fsx = 1.0 / ((mag_samp * mags[m].first) * M->D);
                        const double fsy = 1.0 / ((mag_samp * mags[m].second) * M->D);
                        for (long k = 0; k < nd[t]; ++k) {
                            ImgCtf C = M->h_ictf[P.img];
                            if (dsearch) {
                                C.c[1] = dz.abw20(P.dvals[k]);
                                C.apply = dz.defocus(C.c[1]) >= 1 ? 1 : 0;
                            }
                            C.fsx = fsx;
                            C.fsy = fsy;
                            recs.push_back(C);
                        }
                    }
                }
                e = cudaMemcpyAsync(d_mrec, recs.data(), sizeof(ImgCtf) * recs.size(), cudaMemcpyHostToDevice, s);
                if (e == cudaSuccess) e = launch_ctf_rows(*M, d_mrec, (long)recs.size(), d_mctf, s);
                if (e != cudaSuccess) { r = match_fail(BSG_ERR_CUDA, "bsg_match_refine: %s", cudaGetErrorString(e)); break; }
            }
            const float* table = need_rows ? d_mctf : nullptr;
            auto mgroup = [&](long t, long m) {
                const Particle& P = parts[p0 + t];
                MHypG g;
                memset(&g, 0, sizeof(g));
                memcpy(g.m, &mm[9 * (t * nmag + m)], sizeof(g.m));
                g.img = (int)P.img;
                g.ctf = need_rows ? (int)(rowbase[t] + m * nd[t] + nd[t] - 1) : (int)P.img;
                g.sec = (int)(t * nmag + m);
                return g;
            };
            // pass A: the fits' defocus trials at the best origin
            std::vector<int> vk(np_ * nmag);
            std::vector<double> vfom(np_ * nmag, -1.0), vcv(np_ * nmag, 0.0);
            for (long t = 0; t < np_; ++t)
                for (long m = 0; m < nmag; ++m) vk[t * nmag + m] = (int)nd[t] - 1;
            if (dsearch) {
                groups.clear();
                gfirst.clear();
                for (long t = 0; t < np_; ++t) {
                    const Particle& P = parts[p0 + t];
                    gfirst.push_back((long)groups.size());
                    for (long m = 0; m < nmag; ++m) {
                        MHypG g = mgroup(t, m);
                        g.norg = 1;
                        g.sx[0] = slope(P.box);
                        g.sy[0] = slope(P.boy);
                        for (long k = 0; k + 1 < nd[t]; ++k) {
                            g.ctf = (int)(rowbase[t] + m * nd[t] + k);
                            groups.push_back(g);
                        }
                    }
                }
                r = score_with(table, d_msec);
                if (r != BSG_OK) break;
                for (long t = 0; t < np_; ++t) {
                    Particle& P = parts[p0 + t];
                    const long ntr = nd[t] - 1;
                    for (long m = 0; m < nmag; ++m)
                        for (long k = 0; k < ntr; ++k) {
                            const long g = gfirst[t] + m * ntr + k;
                            const double f = go[g * MAXORG];
                            P.number++;
                            if (vfom[t * nmag + m] < f) {
                                vfom[t * nmag + m] = f;
                                vk[t * nmag + m] = (int)k;
                                vcv[t * nmag + m] = go[(long)groups.size() * MAXORG + g * MAXORG];
                            }
                        }
                }
            }
            // pass B: the shift levels with each fit's chosen defocus
            groups.clear();
            const int nml = (int)mag_steps.size();
            for (long t = 0; t < np_; ++t)
                for (long m = 0; m < nmag; ++m) {
                    MHypG g = mgroup(t, m);
                    if (need_rows) g.ctf = (int)(rowbase[t] + m * nd[t] + vk[t * nmag + m]);
                    for (int k = 0; k < nml; ++k) {
                        const Level& L = lev[t][k];
                        g.norg = L.n;
                        for (int o = 0; o < L.n; ++o) {
                            g.sx[o] = slope(L.x[o]);
                            g.sy[o] = slope(L.y[o]);
                        }
                        groups.push_back(g);
                    }
                }
            r = score_with(table, d_msec);
            if (r != BSG_OK) break;
            const long ng = (long)groups.size();
            const double* gfom = go.data();
            const double* gcv = go.data() + ng * MAXORG;
            for (long t = 0; t < np_; ++t) {
                Particle& P = parts[p0 + t];
                const DefocusTerm dz(dsearch ? M->h_volt[P.img] : 0.0);
                double best = -1, bcv = P.bestcv, bx = P.box, by = P.boy, bdef = P.bestdef, bmx = 1, bmy = 1;
                bool won = false;
                for (long m = 0; m < nmag; ++m) {
                    const long q = t * nmag + m;
                    double fbest = vfom[q], prevfom, fcv = vcv[q], fx = P.box, fy = P.boy;
                    int k = 0;
                    while (k < nml) {
                        const Level& L = lev[t][k];
                        const long g = q * nml + k;
                        prevfom = fbest;
                        fbest = -1;
                        int ib = 0;
                        for (int o = 0; o < L.n; ++o) {
                            const double f = gfom[g * MAXORG + o];
                            P.number++;
                            if (fbest < f) {
                                fbest = f;
                                ib = o;
                                fx = L.x[o];
                                fy = L.y[o];
                                fcv = gcv[g * MAXORG + o];
                            }
                        }
                        if (ib == L.n / 2 || fabs(prevfom - fbest) < 1e-6) ++k;
                    }
                    if (best < fbest) {
                        best = fbest;
                        won = true;
                        bmx = mags[m].first;
                        bmy = mags[m].second;
                        bx = fx;
                        by = fy;
                        bcv = fcv;
                        if (dsearch) bdef = dz.defocus(dz.abw20(P.dvals[vk[q]]));
                    }
                }
                P.bestfom = best;
                if (won) {
                    P.bmx = bmx;
                    P.bmy = bmy;
                    P.box = bx;
                    P.boy = by;
                    P.bestcv = bcv;
                    P.bestdef = bdef;
                }
            }
        }
        cudaFree(d_mm);
        cudaFree(d_msec);
        cudaFree(d_mctf);
        cudaFree(d_mrec);
        return r;
    };

    for (long c0 = 0; c0 < nstart && rc == BSG_OK; c0 += chunk) {
        const long c1 = std::min(nstart, c0 + chunk);
        if (dsearch) {
            // CTF rows of every defocus trial of this chunk's particles
            std::vector<ImgCtf> recs;
            for (long i = c0; i < c1; ++i) {
                Particle& P = parts[i];
                P.row0 = (long)recs.size();
                const DefocusTerm dz(M->h_volt[P.img]);
                for (double d : P.dvals) {
                    ImgCtf C = M->h_ictf[P.img];
                    C.c[1] = dz.abw20(d);
                    // APPLY_CTF is set with -defocus (mg_refine.cpp:575); the
                    // figure of merit drops the CTF below 1 angstrom (:685-686)
                    C.apply = dz.defocus(C.c[1]) >= 1 ? 1 : 0;
                    recs.push_back(C);
                }
            }
            cudaFree(d_rctf);
            cudaFree(d_rrec);
            d_rctf = nullptr;
            d_rrec = nullptr;
            ce = cudaMalloc(&d_rctf, sizeof(float) * npix * recs.size());
            if (ce == cudaSuccess) ce = cudaMalloc(&d_rrec, sizeof(ImgCtf) * recs.size());
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(d_rrec, recs.data(), sizeof(ImgCtf) * recs.size(), cudaMemcpyHostToDevice, s);
            if (ce == cudaSuccess) ce = launch_ctf_rows(*M, d_rrec, (long)recs.size(), d_rctf, s);
            if (ce != cudaSuccess) {
                rc = match_fail(BSG_ERR_CUDA, "bsg_match_refine: %s", cudaGetErrorString(ce));
                break;
            }
        }
        for (;;) {
            owner.clear();
            for (long i = c0; i < c1; ++i) {
                Particle& P = parts[i];
                if (P.done) continue;
                const int nv = views_for_refinement(renormalised(P.bestview, 1), P.alpha, P.views);
                if (nv != NVIEW) {
                    rc = match_fail(BSG_ERR_STATE, "bsg_match_refine: %d refinement views", nv);
                    break;
                }
                owner.push_back(i);
            }
            if (rc != BSG_OK || owner.empty()) break;
            // the views' matrices and their sections, gathered once
            mats.assign(9 * owner.size() * NVIEW, 0.0);
            for (size_t t = 0; t < owner.size(); ++t)
                for (int v = 0; v < NVIEW; ++v) {
                    // Bimage::view stores a twice-copied view; the fit reads
                    // it back (one more) and View::matrix normalises once more
                    double mat[9];
                    view_matrix(renormalised(parts[owner[t]].views[v], 3), mat);
                    match_view_rows(*M, mat, &mats[9 * (t * NVIEW + v)]);
                }
            {
                const long nv = (long)owner.size() * NVIEW;
                cudaError_t e = cudaMemcpyAsync(d_rmats, mats.data(), sizeof(double) * 9 * nv, cudaMemcpyHostToDevice, s);
                if (e == cudaSuccess) e = cudaEventRecord(e0, s);
                if (e == cudaSuccess) e = launch_secgather(*M, d_rmats, nv, d_sec, s);
                if (e == cudaSuccess) e = cudaEventRecord(e1, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) {
                    rc = match_fail(BSG_ERR_CUDA, "bsg_match_refine: %s", cudaGetErrorString(e));
                    break;
                }
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                tsum += ms;
                ++launches;
            }
            // pass A: the fit's defocus trials at the original origin
            // (img_fit_in_recip_space_grid :895-911)
            for (long i : owner)
                for (int v = 0; v < NVIEW; ++v) {
                    parts[i].vk[v] = (int)parts[i].dvals.size() - 1;
                    parts[i].vfom[v] = -1;
                    parts[i].vcv[v] = 0;
                }
            if (dsearch) {
                groups.clear();
                gfirst.clear();
                for (size_t t = 0; t < owner.size(); ++t) {
                    Particle& P = parts[owner[t]];
                    gfirst.push_back((long)groups.size());
                    for (int v = 0; v < NVIEW; ++v) {
                        MHypG g = view_group(P, (long)t, v);
                        g.norg = 1;
                        g.sx[0] = slope(P.ox);
                        g.sy[0] = slope(P.oy);
                        for (size_t k = 0; k + 1 < P.dvals.size(); ++k) {
                            g.ctf = (int)(P.row0 + (long)k);
                            groups.push_back(g);
                        }
                    }
                }
                rc = score(d_rctf);
                if (rc != BSG_OK) break;
                for (size_t t = 0; t < owner.size(); ++t) {
                    Particle& P = parts[owner[t]];
                    const long nd = (long)P.dvals.size() - 1;
                    for (int v = 0; v < NVIEW; ++v)
                        for (long k = 0; k < nd; ++k) {
                            const long g = gfirst[t] + (long)v * nd + k;
                            const double f = go[g * MAXORG];
                            P.number++;
                            if (P.vfom[v] < f) {
                                P.vfom[v] = f;
                                P.vk[v] = (int)k;
                                P.vcv[v] = go[(long)groups.size() * MAXORG + g * MAXORG];
                            }
                        }
                }
            }
            // pass B: every shift level of every view (:914-944), with the
            // defocus each view's trials chose
            groups.clear();
            for (size_t t = 0; t < owner.size(); ++t) {
                Particle& P = parts[owner[t]];
                for (int v = 0; v < NVIEW; ++v) {
                    MHypG g = view_group(P, (long)t, v);
                    if (dsearch) g.ctf = (int)(P.row0 + P.vk[v]);
                    for (int k = 0; k < nlev; ++k) {
                        const Level& L = P.levels[k];
                        g.norg = L.n;
                        for (int o = 0; o < L.n; ++o) {
                            g.sx[o] = slope(L.x[o]);
                            g.sy[o] = slope(L.y[o]);
                        }
                        groups.push_back(g);
                    }
                }
            }
            if (!groups.empty()) {
                rc = score(dsearch ? d_rctf : nullptr);
                if (rc != BSG_OK) break;
            }
            const long ng = (long)groups.size();
            const double* gfom = go.data();
            const double* gcv = go.data() + ng * MAXORG;
            for (size_t t = 0; t < owner.size(); ++t) {
                Particle& P = parts[owner[t]];
                const long gbase = (long)t * NVIEW * nlev;
                const DefocusTerm dz(dsearch ? M->h_volt[P.img] : 0.0);
                // img_refine_grid's angular round (mg_refine.cpp:1112-1136)
                P.prefom = P.bestfom;
                P.bestfom = -1;
                int ibest = 0;
                for (int v = 0; v < NVIEW; ++v) {
                    // img_fit_in_recip_space_grid's shift levels (:914-944),
                    // starting from the defocus trials' best
                    double bestfom = P.vfom[v], prevfom, bestcv = P.vcv[v], bx = P.ox, by = P.oy;
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
                        // the defocus the fit left in the CTF (:1133)
                        if (dsearch) P.bestdef = dz.defocus(dz.abw20(P.dvals[P.vk[v]]));
                    }
                }
                if (ibest == NVIEW / 2 || fabs(P.prefom - P.bestfom) < 1e-6) P.alpha /= 2;
                if (!(P.alpha >= accuracy) || ++P.rounds >= MAX_ROUNDS) P.done = true;
            }
        }
        if (rc == BSG_OK && !mags.empty()) rc = mag_stage(c0, c1);
    }
    cudaFree(d_rctf);
    cudaFree(d_rrec);
    cudaFree(d_rmats);
    cudaFree(d_sec);
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
        o[9] = 0;
        // part->pixel_size = refined sampling x the cut scale (part_refine_orientation,
        // mg_refine.cpp:633): the particle's pixel size after the magnification stage
        o[10] = (mag_samp * P.bmx) * M->cut_scale;
        o[11] = (mag_samp * P.bmy) * M->cut_scale;
        if (dsearch) {
            // the final defocus check (:1186-1191), read back through the CTF
            const DefocusTerm dz(M->h_volt[P.img]);
            const double d = (P.bestdef > P.def0 - 5 * def_std && P.bestdef < P.def0 + 5 * def_std) ? P.bestdef : P.def0;
            o[9] = dz.defocus(dz.abw20(d));
        }
    }
    M->sstats.refine_ms += tsum;
    M->sstats.refine_launches += launches;
    M->sstats.launches += launches;
    return BSG_OK;
}

// ---- brefine -monte: img_refine_monte (mg_refine.cpp:979-1050) with its
// origin/defocus chain img_fit_in_recip_space_monte (:783-860).
//
// The reference draws every random number from the C library's random()
// (seeded once, mg_refine.cpp:276), particle after particle.  Which numbers
// are drawn, and where, never depends on a score, so the host draws each
// start record's whole sequence first, in record order, with glibc's
// generator (random_r on a private TYPE_3 state seeded like srandom): per
// record get_rand_max's 100 draws, then per outer iteration the view step
// (vector3_random_gaussian, random_numbers.cpp:502-510, and the in-plane
// angle), the magnification pair, the fit's own get_rand_max, its defocus
// and origin steps (random_gaussian :123-137, vector3_xy_random_gaussian
// :522-531) and acceptance draws, and the outer acceptance draw.  The
// chains then run in lockstep over all records: one section gather per
// outer iteration, one CTF-row pass and one FP64 figure-of-merit launch per
// inner iteration, and the host applies the reference's acceptance rule
// fom / prefom > u in its order.
namespace bsg {
namespace {

constexpr double TWO_PI_REF = 6.28318530717958647692528676655900576;   // TWOPI (utilities.h)

// the context's random() stream: seed != 0 starts it as srandom(seed)
// does (glibc treats srandom(0) as srandom(1)); 0 continues it
void monte_seed(Match& M, unsigned long long seed) {
    if (seed != 0 || !M.rng_init) {
        memset(&M.rng_data, 0, sizeof(M.rng_data));
        memset(M.rng_state, 0, sizeof(M.rng_state));
        initstate_r(seed != 0 ? (unsigned)seed : 1u, M.rng_state, sizeof(M.rng_state), &M.rng_data);
        M.rng_init = true;
    }
}

long monte_next(Match& M) {
    int32_t r = 0;
    random_r(&M.rng_data, &r);
    return (long)r;
}

struct MonteOuter {
    double r[3] = {0, 0, 0};   // view vector step
    double a = 0;              // in-plane angle step
    double mx = 1, my = 1;     // sampling factors
    double u = 0;              // acceptance draw (random() * irm)
};

struct MonteInner {
    double g = 0;              // defocus step (angstrom)
    double dx = 0, dy = 0;     // origin step (pixels of the cut transform)
    double u = 0;              // acceptance draw
};

struct MonteRec {
    long img = 0;
    bool fit_ctf = false;          // the fit draws defocus steps (flags & APPLY_CTF)
    bool dsearch = false;          // def_std > 0 with a defocus: the defocus chain
    double ox = 0, oy = 0;         // original origin (cut pixels)
    double def0 = 0;               // the particle's defocus
    std::vector<MonteOuter> outer;
    std::vector<MonteInner> inner; // max_iter x max_iter
    // outer chain
    View4 view, preview, bestview;
    double prefom = -1, bestfom = -1, bestcv = 0, bx = 0, by = 0, bestdef = 0, bmx = 1, bmy = 1;
    double mx = 1, my = 1;
    long number = 0;
    // inner chain of the current outer iteration
    double x = 0, y = 0, px = 0, py = 0, fbx = 0, fby = 0;
    double fprefom = -1, fbestfom = -1, fbestcv = 0;
    double abw = 0, pabw = 0, fbestabw = 0;   // CTF abw[2,0] of the current / accepted / best defocus
};

}  // namespace
}  // namespace bsg

extern "C" int bsg_match_refine_monte(bsg_match* h, const double* start, long nstart, int max_iter, double def_std,
                                      double shift_std, double view_std, double max_angle, double max_mag,
                                      unsigned long long seed, double* out, int flags) {
    using namespace bsg;
    const bool dpr = (flags & BSG_MATCH_SCORE_DPR) != 0;
    Match* M = reinterpret_cast<Match*>(h);
    if (!M || !start || !out || nstart < 1) return match_fail(BSG_ERR_ARG, "bsg_match_refine_monte: bad argument");
    if (!M->have_ref || M->nimg < 1)
        return match_fail(BSG_ERR_STATE, "bsg_match_refine_monte: set the reference and images first");
    if (max_iter < 1 || max_iter > 10000)
        return match_fail(BSG_ERR_ARG, "bsg_match_refine_monte: %d iterations outside 1..10000", max_iter);
    if (!(def_std >= 0) || !(shift_std >= 0) || !(view_std >= 0) || !(max_angle >= 0) || !(max_mag >= 0) ||
        !(max_mag < 1) || !isfinite(def_std + shift_std + view_std + max_angle))
        return match_fail(BSG_ERR_ARG, "bsg_match_refine_monte: bad step sizes");
    cudaError_t ce = cudaSetDevice(M->device);
    if (ce != cudaSuccess) return match_fail(BSG_ERR_CUDA, "bsg_match_refine_monte: %s", cudaGetErrorString(ce));

    // ---- the random draws, record after record (the reference's order)
    monte_seed(*M, seed);
    auto rnd = [&]() { return monte_next(*M); };
    auto get_rand_max = [&]() {          // random_numbers.cpp:22-30
        long rm = 32767;
        for (int i = 0; i < 100; ++i)
            if (rnd() > rm) rm = 2147483647;
        return rm;
    };
    // random_numbers.cpp's file-scope irm = 1.0L / get_rand_max(), formed
    // before main from the unseeded generator: 2^31 - 1 for 31-bit random()
    const double girm = (double)(1.0L / 2147483647.0L);
    auto gauss = [&](double avg, double sd) {
        double r = -2 * log(rnd() * girm);
        if (r > 0) r = avg + sd * sqrt(r) * cos(TWO_PI_REF * (rnd() * girm));
        else r = avg;
        return r;
    };
    const long ni = (long)max_iter;
    std::vector<MonteRec> recs(nstart);
    for (long i = 0; i < nstart; ++i) {
        const double* r = start + BSG_MATCH_REFINE_START_DOUBLES * i;
        const long img = (long)r[0];
        if (!(r[0] >= 0) || img >= M->nimg)
            return match_fail(BSG_ERR_ARG, "bsg_match_refine_monte: start record %ld names image %g", i, r[0]);
        MonteRec& R = recs[i];
        R.img = img;
        R.ox = M->cut_scale * r[5];
        R.oy = M->cut_scale * r[6];
        R.view = R.preview = R.bestview = renormalised(make_view(r[1], r[2], r[3], r[4]), 3);
        R.bx = R.ox;
        R.by = R.oy;
        R.dsearch = def_std > 0;
        R.fit_ctf = R.dsearch || M->h_ictf[img].apply;
        if (R.fit_ctf && !(M->h_volt[img] > 0))
            return match_fail(BSG_ERR_ARG, "bsg_match_refine_monte: image %ld has a CTF but no voltage", img);
        if (R.dsearch) {
            const DefocusTerm dz(M->h_volt[img]);
            R.def0 = dz.defocus(M->h_ictf[img].c[1]);
            if (R.def0 == 0)
                return match_fail(BSG_ERR_ARG, "bsg_match_refine_monte: image %ld has no defocus to vary", img);
        }
        R.bestdef = R.def0;
        R.outer.resize(ni);
        R.inner.resize(ni * ni);
        const double irm = 1.0 / get_rand_max();              // img_refine_monte's irm
        for (long o = 0; o < ni; ++o) {
            MonteOuter& od = R.outer[o];
            if (o > 0) {
                // vector3_random_gaussian: a unit vector (3 gaussians), then the length
                Vec3 u{{gauss(0, 1), gauss(0, 1), gauss(0, 1)}};
                u.normalize();
                const double amp = gauss(0, view_std);
                for (int k = 0; k < 3; ++k) od.r[k] = u.d[k] * amp;
                od.a = max_angle * (rnd() * irm * 2 - 1);
                if (max_mag > 0) {
                    od.mx = 1 + max_mag * (rnd() * irm * 2 - 1);
                    od.my = 1 + max_mag * (rnd() * irm * 2 - 1);
                }
            }
            const double firm = 1.0 / get_rand_max();         // the fit's irm
            for (long it = 0; it < ni; ++it) {
                MonteInner& id = R.inner[o * ni + it];
                if (it > 0) {
                    if (R.fit_ctf) id.g = gauss(0, def_std);
                    // vector3_xy_random_gaussian: the length first, then x and y
                    const double amp = gauss(0, shift_std);
                    Vec3 v{{gauss(0, 1), gauss(0, 1), 0}};
                    v.normalize();
                    id.dx = v.d[0] * amp;
                    id.dy = v.d[1] * amp;
                }
                id.u = rnd() * firm;
            }
            od.u = rnd() * irm;
        }
    }

    // ---- the chains, all records in lockstep
    const int npix = (int)M->h_pix.size();
    const double mag_samp = M->cfg.pixel / M->cut_scale;
    const double ref_samp = M->cfg.map_sampling / (double)((long double)M->D / M->N);
    const long cap = std::max(1L, std::min(nstart, (long)((1L << 30) / ((long)sizeof(double2) * std::max(npix, 1)))));
    cudaStream_t s = M->stream;
    double* d_mats = nullptr;
    double2* d_sec = nullptr;
    float* d_ctfrows = nullptr;
    ImgCtf* d_crec = nullptr;
    ce = cudaMalloc(&d_mats, sizeof(double) * 9 * cap);
    if (ce == cudaSuccess) ce = cudaMalloc(&d_sec, sizeof(double2) * (size_t)npix * cap);
    if (ce == cudaSuccess) ce = cudaMalloc(&d_ctfrows, sizeof(float) * (size_t)npix * cap);
    if (ce == cudaSuccess) ce = cudaMalloc(&d_crec, sizeof(ImgCtf) * cap);
    int rc = BSG_OK;
    if (ce != cudaSuccess) rc = match_fail(BSG_ERR_NOMEM, "bsg_match_refine_monte: %s", cudaGetErrorString(ce));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float tsum = 0;
    long launches = 0;
    auto slope = [&](double o) { return o / M->D * 2 * M_PI; };
    std::vector<double> mats;
    std::vector<MHypG> groups;
    std::vector<ImgCtf> crec;
    std::vector<double> go;
    for (long c0 = 0; c0 < nstart && rc == BSG_OK; c0 += cap) {
        const long c1 = std::min(nstart, c0 + cap), nc = c1 - c0;
        for (long o = 0; o < ni && rc == BSG_OK; ++o) {
            // the outer step: view, sampling; p->view(view) stores a copy the fit reads back
            mats.assign(9 * nc, 0.0);
            for (long t = 0; t < nc; ++t) {
                MonteRec& R = recs[c0 + t];
                const MonteOuter& od = R.outer[o];
                if (o > 0) {
                    R.view.v[0] += od.r[0];
                    R.view.v[1] += od.r[1];
                    R.view.v[2] += od.r[2];
                    R.view.a += od.a;
                    R.view.normalize();
                    R.mx = od.mx;
                    R.my = od.my;
                }
                double mat[9];
                view_matrix(renormalised(R.view, 3), mat);
                const double kx = ref_samp / (mag_samp * R.mx), ky = ref_samp / (mag_samp * R.my);
                double* mo = &mats[9 * t];
                for (int a = 0; a < 3; ++a)
                    for (int c = 0; c < 3; ++c) {
                        double v = mat[3 * a + c];
                        if (a < 2) v *= (c == 0 ? kx : (c == 1 ? ky : 1.0));
                        mo[3 * a + c] = v;
                    }
                // the fit starts from the original origin and defocus
                R.x = R.px = R.fbx = R.ox;
                R.y = R.py = R.fby = R.oy;
                R.fprefom = -1;
                R.fbestfom = -1;
                R.fbestcv = 0;
                if (R.dsearch) {
                    const DefocusTerm dz(M->h_volt[R.img]);
                    R.abw = R.pabw = R.fbestabw = dz.abw20(R.def0);
                } else {
                    R.abw = R.pabw = R.fbestabw = M->h_ictf[R.img].c[1];
                }
            }
            cudaError_t e = cudaMemcpyAsync(d_mats, mats.data(), sizeof(double) * mats.size(), cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaEventRecord(e0, s);
            if (e == cudaSuccess) e = launch_secgather(*M, d_mats, nc, d_sec, s);
            if (e == cudaSuccess) e = cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) { rc = match_fail(BSG_ERR_CUDA, "bsg_match_refine_monte: %s", cudaGetErrorString(e)); break; }
            {
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                tsum += ms;
                ++launches;
            }
            for (long it = 0; it < ni; ++it) {
                groups.assign(nc, MHypG{});
                crec.resize(nc);
                for (long t = 0; t < nc; ++t) {
                    MonteRec& R = recs[c0 + t];
                    const MonteInner& id = R.inner[o * ni + it];
                    if (it > 0) {
                        if (R.fit_ctf) {
                            // em_ctf->defocus_average(em_ctf->defocus_average() + g)
                            const DefocusTerm dz(M->h_volt[R.img]);
                            R.abw = dz.abw20(dz.defocus(R.abw) + id.g);
                        }
                        R.x += id.dx;
                        R.y += id.dy;
                    }
                    MHypG& g = groups[t];
                    memset(&g, 0, sizeof(g));
                    memcpy(g.m, &mats[9 * t], sizeof(g.m));
                    g.img = (int)R.img;
                    g.ctf = (int)t;
                    g.sec = (int)t;
                    g.norg = 1;
                    g.sx[0] = slope(R.x);
                    g.sy[0] = slope(R.y);
                    ImgCtf C = M->h_ictf[R.img];
                    if (R.fit_ctf) {
                        C.c[1] = R.abw;
                        if (R.dsearch) {
                            const DefocusTerm dz(M->h_volt[R.img]);
                            C.apply = dz.defocus(C.c[1]) >= 1 ? 1 : 0;
                        }
                    }
                    C.fsx = 1.0 / ((mag_samp * R.mx) * M->D);
                    C.fsy = 1.0 / ((mag_samp * R.my) * M->D);
                    crec[t] = C;
                }
                const long ng = nc;
                int r2 = ensure_groups(*M, ng);
                if (r2 != BSG_OK) { rc = r2; break; }
                go.resize(2 * ng * MAXORG);
                e = cudaMemcpyAsync(M->d_grp, groups.data(), sizeof(MHypG) * ng, cudaMemcpyHostToDevice, s);
                if (e == cudaSuccess) e = cudaMemcpyAsync(d_crec, crec.data(), sizeof(ImgCtf) * nc, cudaMemcpyHostToDevice, s);
                if (e == cudaSuccess) e = cudaEventRecord(e0, s);
                if (e == cudaSuccess) e = launch_ctf_rows(*M, d_crec, nc, d_ctfrows, s);
                if (e == cudaSuccess)
                    e = launch_fom(*M, M->d_grp, ng, M->d_gout, M->d_gout + ng * MAXORG, s, true, d_ctfrows, d_sec, dpr);
                if (e == cudaSuccess) e = cudaEventRecord(e1, s);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(go.data(), M->d_gout, sizeof(double) * go.size(), cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) { rc = match_fail(BSG_ERR_CUDA, "bsg_match_refine_monte: %s", cudaGetErrorString(e)); break; }
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                tsum += ms;
                launches += 2;
                // img_fit_in_recip_space_monte's bookkeeping (:827-850)
                for (long t = 0; t < nc; ++t) {
                    MonteRec& R = recs[c0 + t];
                    const MonteInner& id = R.inner[o * ni + it];
                    double fom = go[t * MAXORG];
                    const double cv = go[ng * MAXORG + t * MAXORG];
                    R.number++;
                    if (R.fbestfom < fom) {
                        R.fbestfom = fom;
                        R.fbestabw = R.abw;
                        R.fbx = R.x;
                        R.fby = R.y;
                        R.fbestcv = cv;
                    }
                    if (fom / R.fprefom > id.u) {
                        R.pabw = R.abw;
                        R.px = R.x;
                        R.py = R.y;
                        R.fprefom = fom;
                    } else {
                        R.abw = R.pabw;
                        R.x = R.px;
                        R.y = R.py;
                    }
                }
            }
            if (rc != BSG_OK) break;
            // img_refine_monte's bookkeeping (:1025-1046)
            for (long t = 0; t < nc; ++t) {
                MonteRec& R = recs[c0 + t];
                const double fom = R.fbestfom;
                if (R.bestfom < fom) {
                    R.bestfom = fom;
                    R.bestview = R.view;
                    R.bmx = R.mx;
                    R.bmy = R.my;
                    R.bx = R.fbx;
                    R.by = R.fby;
                    if (R.dsearch) {
                        const DefocusTerm dz(M->h_volt[R.img]);
                        R.bestdef = dz.defocus(R.fbestabw);
                    }
                    R.bestcv = R.fbestcv;
                }
                if (fom / R.prefom > R.outer[o].u) {
                    R.preview = R.view;
                    R.prefom = fom;
                } else {
                    R.view = R.preview;
                }
            }
        }
    }
    cudaFree(d_mats);
    cudaFree(d_sec);
    cudaFree(d_ctfrows);
    cudaFree(d_crec);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != BSG_OK) return rc;
    for (long i = 0; i < nstart; ++i) {
        const MonteRec& R = recs[i];
        const View4 w = renormalised(R.bestview, 3);
        double* o = out + BSG_MATCH_REFINE_RESULT_DOUBLES * i;
        o[0] = w.v[0];
        o[1] = w.v[1];
        o[2] = w.v[2];
        o[3] = w.a;
        o[4] = R.bx / M->cut_scale;
        o[5] = R.by / M->cut_scale;
        o[6] = R.bestfom;
        o[7] = R.bestcv;
        o[8] = (double)R.number;
        o[9] = R.dsearch ? R.bestdef : 0.0;
        o[10] = (mag_samp * R.bmx) * M->cut_scale;
        o[11] = (mag_samp * R.bmy) * M->cut_scale;
    }
    M->sstats.refine_ms += tsum;
    M->sstats.refine_launches += launches;
    M->sstats.launches += launches;
    return BSG_OK;
}
