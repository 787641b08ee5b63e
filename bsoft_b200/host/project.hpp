// project.hpp - host-side readers and writers shared by the drop-in
// executables (breconstruct.cpp, brefine.cpp): STAR parameter files (the
// syntax of bsoft/src/util/rwstar.cpp), MRC images (bsoft/src/rwimg/
// rwMRC.cpp:60-215), the micrograph / particle project model of
// read_project (rwmgSTAR.cpp:195-262, 458-519, 521-655; rwmg.cpp:650-659),
// the view -> matrix convention (View.h, Matrix3.h) and the CTF aberration
// weights (ctf.h).
#pragma once

#include <array>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace bsh {

// ---------------------------------------------------------------- STAR
struct StarLoop {
    std::vector<std::string> tags;
    std::vector<std::vector<std::string>> rows;
    int index(const std::string& t) const {
        for (size_t i = 0; i < tags.size(); ++i)
            if (tags[i] == t) return (int)i;
        return -1;
    }
};

struct StarBlock {
    std::string name;
    std::map<std::string, std::string> items;
    std::vector<StarLoop> loops;
    bool has(const std::string& t) const { return items.count(t) > 0; }
    double real(const std::string& t, double def = 0) const {
        auto it = items.find(t);
        if (it == items.end()) return def;
        char* end = nullptr;
        const double v = strtod(it->second.c_str(), &end);
        return end == it->second.c_str() ? def : v;
    }
    long integer(const std::string& t, long def = 0) const { return (long)real(t, (double)def); }
    const StarLoop* loop_with(const std::string& t) const {
        for (auto& l : loops)
            if (l.index(t) >= 0) return &l;
        return nullptr;
    }
};

// whitespace-separated tokens; single or double quotes group
inline std::vector<std::string> tokens(const std::string& line) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < line.size()) {
        while (i < line.size() && isspace((unsigned char)line[i])) ++i;
        if (i >= line.size()) break;
        if (line[i] == '\'' || line[i] == '"') {
            const char q = line[i++];
            size_t j = line.find(q, i);
            if (j == std::string::npos) j = line.size();
            out.push_back(line.substr(i, j - i));
            i = j + 1;
        } else {
            size_t j = i;
            while (j < line.size() && !isspace((unsigned char)line[j])) ++j;
            out.push_back(line.substr(i, j - i));
            i = j;
        }
    }
    return out;
}

inline std::vector<StarBlock> read_star(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::vector<StarBlock> blocks;
    StarLoop* loop = nullptr;
    bool in_header = false;
    std::string raw;
    while (std::getline(f, raw)) {
        size_t a = raw.find_first_not_of(" \t\r\n");
        const std::string line = a == std::string::npos ? "" : raw.substr(a, raw.find_last_not_of(" \t\r\n") - a + 1);
        if (line.empty() || line[0] == '#') {
            if (line.empty() && loop && !in_header && !loop->rows.empty()) loop = nullptr;
            continue;
        }
        if (line.compare(0, 5, "data_") == 0) {
            blocks.push_back(StarBlock{line.substr(5), {}, {}});
            loop = nullptr;
            continue;
        }
        if (blocks.empty()) continue;
        StarBlock& cur = blocks.back();
        if (line.compare(0, 5, "loop_") == 0) {
            cur.loops.emplace_back();
            loop = &cur.loops.back();
            in_header = true;
            continue;
        }
        if (line[0] == '_') {
            if (loop && in_header) {
                loop->tags.push_back(tokens(line)[0].substr(1));
                continue;
            }
            loop = nullptr;
            auto t = tokens(line);
            cur.items[t[0].substr(1)] = t.size() > 1 ? t[1] : "";
            continue;
        }
        if (loop) {
            in_header = false;
            auto t = tokens(line);
            if (t.size() == loop->tags.size()) loop->rows.push_back(t);
        }
    }
    return blocks;
}

// ---------------------------------------------------------------- MRC
struct MrcHeader {
    int nx = 0, ny = 0, nz = 0, mode = 0, mx = 0, my = 0, mz = 0, nsymbt = 0, nversion = 0;
    float cell[3] = {0, 0, 0}, origin[3] = {0, 0, 0};
    float dmean = 0, rms = 0;        // header statistics (rwMRC.cpp:181-184)
    double sampling(int i) const {
        const int m = i == 0 ? (mx ? mx : 1) : i == 1 ? (my ? my : 1) : (mz ? mz : 1);
        return cell[i] ? cell[i] / m : 1.0;
    }
    long images() const { return (nversion >= 20140 && nversion <= 20209 && mz) ? nz / mz : nz; }
    // rwMRC.cpp:195: image origin (pixels) = -origin field / sampling
    double image_origin(int i) const { return -origin[i] / sampling(i); }
};

inline MrcHeader read_mrc_header(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    unsigned char raw[1024];
    if (!f.read((char*)raw, 1024)) throw std::runtime_error(path + ": short MRC header");
    MrcHeader h;
    int32_t iv[10];
    memcpy(iv, raw, 40);
    h.nx = iv[0]; h.ny = iv[1]; h.nz = iv[2]; h.mode = iv[3]; h.mx = iv[7]; h.my = iv[8]; h.mz = iv[9];
    memcpy(h.cell, raw + 40, 12);
    memcpy(&h.nsymbt, raw + 92, 4);
    memcpy(&h.nversion, raw + 108, 4);
    memcpy(h.origin, raw + 196, 12);
    memcpy(&h.dmean, raw + 84, 4);
    memcpy(&h.rms, raw + 216, 4);
    if (h.nx < 1 || h.ny < 1 || h.nz < 1 || h.mode < 0 || h.mode > 16)
        throw std::runtime_error(path + ": not a valid little-endian MRC image");
    return h;
}

// float32 images [first, first + count) of a mode-2 stack
inline void read_mrc_images(const std::string& path, const MrcHeader& h, long first, long count, float* out) {
    if (h.mode != 2) throw std::runtime_error(path + ": only mode 2 (float32) stacks are supported");
    const long per = (long)h.nx * h.ny * ((h.nversion >= 20140 && h.mz) ? h.mz : 1);
    if (first < 0 || first + count > h.images()) throw std::runtime_error(path + ": image index outside the stack");
    std::ifstream f(path, std::ios::binary);
    f.seekg(1024 + (long)h.nsymbt + first * per * 4);
    if (!f.read((char*)out, sizeof(float) * per * count)) throw std::runtime_error(path + ": truncated data");
}

// a whole mode-2 volume (nx x ny x nz floats, x fastest)
inline std::vector<float> read_mrc_volume(const std::string& path, const MrcHeader& h) {
    if (h.mode != 2) throw std::runtime_error(path + ": only mode 2 (float32) maps are supported");
    std::vector<float> v((size_t)h.nx * h.ny * h.nz);
    std::ifstream f(path, std::ios::binary);
    f.seekg(1024 + (long)h.nsymbt);
    if (!f.read((char*)v.data(), sizeof(float) * v.size())) throw std::runtime_error(path + ": truncated data");
    return v;
}

// ---------------------------------------------------------------- SPIDER
// Real-space float stacks as the reference's SPIDER reader reads them
// (bsoft/src/rwimg/rwSPIDER.cpp:82-243): header words as floats (nslice 0,
// nrow 1, iform 4, av 8, sig 9, nsam 11, xoff/yoff/zoff 17-19, scale 20,
// labbyt 21, istack 23, maxim 25); the words (and the data) are byte-swapped
// when |nslice| or |iform| exceeds 65535 or |nslice| < 1; a stack
// (istack > 0) holds maxim images, image i being a labbyt-byte header and
// its data at labbyt + i (labbyt + 4 nsam nrow nslice); sampling = scale;
// each image's origin is its own header's.
struct SpiderHeader {
    int nx = 0, ny = 0, nz = 0;
    float iform = 0, istack = 0, scale = 1, av = 0, sig = 0;
    long labbyt = 0, maxim = 0;
    bool swap = false;
    std::vector<double> ox, oy;      // per image origin (pixels)
    long images() const { return istack > 0 ? maxim : 1; }
    long image_bytes() const { return labbyt + 4L * nx * ny * nz; }
    long data_offset(long i) const { return istack > 0 ? labbyt + i * image_bytes() + labbyt : labbyt; }
};

inline bool is_spider(const std::string& path) {
    auto ends = [&](const char* e) {
        const size_t n = strlen(e);
        if (path.size() < n) return false;
        for (size_t i = 0; i < n; ++i)
            if (tolower((unsigned char)path[path.size() - n + i]) != e[i]) return false;
        return true;
    };
    return ends(".spi") || ends(".spider");
}

inline void spider_words(const unsigned char* raw, bool swap, float* w) {
    for (int i = 0; i < 36; ++i) {
        unsigned char b[4] = {raw[4 * i], raw[4 * i + 1], raw[4 * i + 2], raw[4 * i + 3]};
        if (swap) { std::swap(b[0], b[3]); std::swap(b[1], b[2]); }
        memcpy(&w[i], b, 4);
    }
}

inline SpiderHeader read_spider_header(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    unsigned char raw[1024];
    if (!f.read((char*)raw, 1024)) throw std::runtime_error(path + ": short SPIDER header");
    float w[36];
    spider_words(raw, false, w);
    SpiderHeader h;
    h.swap = fabsf(w[0]) > 65535 || fabsf(w[4]) > 65535 || fabsf(w[0]) < 1;
    if (h.swap) spider_words(raw, true, w);
    h.nz = (int)w[0]; h.ny = (int)w[1]; h.nx = (int)w[11];
    h.iform = w[4]; h.av = w[8]; h.sig = w[9]; h.scale = w[20];
    h.labbyt = (long)w[21]; h.istack = w[23]; h.maxim = (long)w[25];
    if (h.nx < 1 || h.ny < 1 || h.nz < 1 || h.labbyt < 144)
        throw std::runtime_error(path + ": not a valid SPIDER image");
    if (h.iform < 0) throw std::runtime_error(path + ": SPIDER Fourier transforms are not particle stacks");
    const long n = h.images();
    h.ox.assign(n, w[17]);
    h.oy.assign(n, w[18]);
    if (h.istack > 0)
        for (long i = 0; i < n; ++i) {
            f.seekg(h.labbyt + i * h.image_bytes());
            if (!f.read((char*)raw, 144)) throw std::runtime_error(path + ": truncated image header");
            spider_words(raw, h.swap, w);
            h.ox[i] = w[17];
            h.oy[i] = w[18];
        }
    return h;
}

inline void read_spider_images(const std::string& path, const SpiderHeader& h, long first, long count, float* out) {
    if (first < 0 || first + count > h.images()) throw std::runtime_error(path + ": image index outside the stack");
    const long per = (long)h.nx * h.ny * h.nz;
    std::ifstream f(path, std::ios::binary);
    for (long j = 0; j < count; ++j) {
        f.seekg(h.data_offset(first + j));
        float* o = out + j * per;
        if (!f.read((char*)o, sizeof(float) * per)) throw std::runtime_error(path + ": truncated data");
        if (h.swap)
            for (long k = 0; k < per; ++k) {
                unsigned char* b = (unsigned char*)(o + k);
                std::swap(b[0], b[3]);
                std::swap(b[1], b[2]);
            }
    }
}

// ---------------------------------------------------------------- stacks
// Particle stacks by format, as read_img picks the reader from the file
// extension (bsoft/src/rwimg/rwimg.cpp:79-130): .spi / .spider -> SPIDER,
// else MRC.
struct StackHeader {
    bool spider = false;
    MrcHeader mrc;
    SpiderHeader spi;
    int nx() const { return spider ? spi.nx : mrc.nx; }
    int ny() const { return spider ? spi.ny : mrc.ny; }
    double sampling(int i) const { return spider ? (double)spi.scale : mrc.sampling(i); }
    long images() const { return spider ? spi.images() : mrc.images(); }
    // origin (pixels) of image img: the MRC header's for every image, a
    // SPIDER stack's per image
    double image_origin(int axis, long img) const {
        if (!spider) return mrc.image_origin(axis);
        const std::vector<double>& v = axis == 0 ? spi.ox : spi.oy;
        return v.empty() ? 0.0 : v[std::min<long>(std::max<long>(img, 0), (long)v.size() - 1)];
    }
    // the file statistics read_img attaches (MRC dmean/rms, SPIDER av/sig)
    double mean() const { return spider ? spi.av : mrc.dmean; }
    double stddev() const { return spider ? spi.sig : mrc.rms; }
};

inline StackHeader read_stack_header(const std::string& path) {
    StackHeader h;
    h.spider = is_spider(path);
    if (h.spider) h.spi = read_spider_header(path);
    else h.mrc = read_mrc_header(path);
    return h;
}

inline void read_stack_images(const std::string& path, const StackHeader& h, long first, long count, float* out) {
    if (h.spider) read_spider_images(path, h.spi, first, count, out);
    else read_mrc_images(path, h.mrc, first, count, out);
}

inline void write_mrc_volume(const std::string& path, const float* v, int N, double sampling, double origin) {
    unsigned char hdr[1024];
    memset(hdr, 0, sizeof(hdr));
    const int32_t iv[10] = {N, N, N, 2, 0, 0, 0, N, N, N};
    memcpy(hdr, iv, 40);
    const float cell[6] = {(float)(N * sampling), (float)(N * sampling), (float)(N * sampling), 90.f, 90.f, 90.f};
    memcpy(hdr + 40, cell, 24);
    const int32_t axes[3] = {1, 2, 3};
    memcpy(hdr + 64, axes, 12);
    const size_t n3 = (size_t)N * N * N;
    double mn = v[0], mx = v[0], sum = 0, sum2 = 0;
    for (size_t i = 0; i < n3; ++i) {
        mn = std::fmin(mn, v[i]);
        mx = std::fmax(mx, v[i]);
        sum += v[i];
        sum2 += (double)v[i] * v[i];
    }
    const double avg = sum / n3, rms = std::sqrt(std::fmax(0.0, sum2 / n3 - avg * avg));
    const float st[3] = {(float)mn, (float)mx, (float)avg};
    memcpy(hdr + 76, st, 12);
    const int32_t ver = 20140;
    memcpy(hdr + 108, &ver, 4);
    const float org[3] = {(float)(-origin * sampling), (float)(-origin * sampling), (float)(-origin * sampling)};
    memcpy(hdr + 196, org, 12);
    memcpy(hdr + 208, "MAP ", 4);
    const unsigned char stamp[4] = {0x44, 0x44, 0, 0};
    memcpy(hdr + 212, stamp, 4);
    const float frms = (float)rms;
    memcpy(hdr + 216, &frms, 4);
    std::ofstream f(path, std::ios::binary);
    f.write((const char*)hdr, 1024);
    f.write((const char*)v, sizeof(float) * n3);
    if (!f) throw std::runtime_error("cannot write " + path);
}

// ---------------------------------------------------------------- geometry and CTF
constexpr double TRIG = 1e-30;   // TRIGPRECISION / SMALLFLOAT

// angle_set_negPI_to_PI (bsoft/src/util/utilities.cpp:606-615)
inline double angle_neg_pi_to_pi(double a) {
    if (!std::isfinite(a)) return 0;
    const long n = (long)(a / M_PI);
    return a - (double)(n + n % 2) * M_PI;
}

// View::normalize + View::quaternion + Matrix3(Quaternion)
// (View.h:110-116, 131-157; Matrix3.h:21-42), row-major
inline void view_matrix(double x, double y, double z, double a, double* m) {
    const double size = std::sqrt(x * x + y * y + z * z);
    if (size < TRIG) { x = 0; y = 0; z = 1; }
    else { x /= size; y /= size; z /= size; }
    if (std::fabs(x) < TRIG) x = 0;
    if (std::fabs(y) < TRIG) y = 0;
    if (std::fabs(z) < TRIG) z = 0;
    a = angle_neg_pi_to_pi(a);
    if (std::fabs(a) < TRIG) a = 0;
    const double ang = a / 2.0, ca = std::cos(ang), sa = std::sin(ang), z1 = z + 1.0;
    double q[4] = {ca, 0, 0, sa};
    if (z < 1.0 - TRIG) {
        if (z <= TRIG - 1.0) {
            q[0] = 0; q[1] = sa; q[2] = ca; q[3] = 0;
        } else {
            const double f1 = std::sqrt(z1 / 2.0), f2 = std::sqrt(1.0 / (2 * z1));
            q[0] = f1 * ca; q[1] = f2 * (x * sa - y * ca); q[2] = f2 * (x * ca + y * sa); q[3] = f1 * sa;
        }
    }
    for (double& t : q)
        if (std::fabs(t) < TRIG) t = 0;
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
        if (std::fabs(m[i]) < 1e-12) m[i] = 0;
        m[i] = std::fmin(1.0, std::fmax(-1.0, m[i]));
    }
}

// CTFparam (bsoft/include/ctf.h): the aberration weights the C ABI takes
struct Ctf {
    double volt = 300000, cs = 2.7e7, amp_shift = 0, defocus = 20000, def_dev = 0, ast_angle = 0;
    double btx = 0, bty = 0;
    // relativistic electron wavelength in angstrom (ctf.h:309-317)
    double lambda() const {
        const double h = 6.626070e-34, me = 9.109384e-31, e = 1.602177e-19, cl = 299792458.0;
        return volt > 0 ? h * 1e10 / std::sqrt(2.0 * me * e * volt * (1.0 + e * volt / (2.0 * me * cl * cl))) : 0;
    }
    void coefficients(double* c) const {
        const double wl = lambda();
        const double t1 = M_PI / 2 * wl * wl * wl, t2 = -M_PI * wl, dev = std::fabs(def_dev);
        c[0] = -amp_shift;
        c[1] = t2 * defocus;
        c[2] = t2 * dev * std::cos(2 * ast_angle);
        c[3] = t2 * dev * std::sin(2 * ast_angle);
        c[4] = t1 * cs;
        c[5] = 2 * M_PI * btx;
        c[6] = 2 * M_PI * bty;
    }
};

// ---------------------------------------------------------------- project
struct Micrograph {
    std::string id, particle_file;
    int box = 0;
    double pixel_size = 0;
    bool has_ctf = false;
    Ctf ctf;
    std::vector<long> part_id;
    std::vector<double> ox, oy, vx, vy, vz, va, defocus, mag, pixel;
    std::vector<double> pixel_y;     // particle pixel size along y (the x one where the file has none)
    std::vector<long> select;
};

inline std::string dir_of(const std::string& p) {
    const size_t s = p.find_last_of('/');
    return s == std::string::npos ? "." : p.substr(0, s);
}

inline std::vector<Micrograph> read_project(const std::string& path) {
    auto blocks = read_star(path);
    const std::string base = dir_of(path);
    std::vector<Micrograph> out;
    for (auto& b : blocks) {
        if (!(b.has("micrograph.id") || b.has("micrograph.file_name"))) continue;
        Micrograph mg;
        mg.id = b.has("micrograph.id") ? b.items.at("micrograph.id") : b.items.at("micrograph.file_name");
        mg.particle_file = b.has("particle.file_name") ? b.items.at("particle.file_name") : "";
        if (!mg.particle_file.empty() && mg.particle_file[0] != '/') mg.particle_file = base + "/" + mg.particle_file;
        // box size vector as micrograph_from_starblock fills it (rwmgSTAR.cpp:590-605)
        long bs[3] = {0, 0, 0};
        if (b.has("particle.box_radius")) bs[0] = bs[1] = bs[2] = 2 * b.integer("particle.box_radius");
        if (b.has("particle.box_radius_x")) {
            bs[0] = 2 * b.integer("particle.box_radius_x"); bs[1] = 2 * b.integer("particle.box_radius_y");
            bs[2] = 2 * b.integer("particle.box_radius_z");
        }
        if (b.has("particle.box_size")) bs[0] = bs[1] = bs[2] = b.integer("particle.box_size");
        if (b.has("particle.box_size_x")) {
            bs[0] = b.integer("particle.box_size_x"); bs[1] = b.integer("particle.box_size_y");
            bs[2] = b.integer("particle.box_size_z");
        }
        mg.box = (int)bs[0];
        mg.pixel_size = b.real("micrograph.pixel_size");
        if (mg.pixel_size == 0) mg.pixel_size = b.real("micrograph.pixel_size_x");
        if (b.has("ctf.voltage")) {
            mg.has_ctf = true;
            Ctf& c = mg.ctf;
            c.amp_shift = b.has("ctf.amplitude_phase_shift") ? b.real("ctf.amplitude_phase_shift")
                                                              : std::asin(b.real("ctf.amp_contrast"));
            if (b.has("ctf.defocus_average")) {
                c.defocus = b.real("ctf.defocus_average");
                c.def_dev = b.real("ctf.defocus_deviation");
            } else {
                const double dmin = b.real("ctf.defocus_min"), dmax = b.real("ctf.defocus_max");
                c.defocus = (dmax + dmin) / 2;
                c.def_dev = std::fabs(dmax - dmin) / 2;
            }
            c.volt = b.real("ctf.voltage");
            if (c.volt < 1e3) c.volt *= 1e3;    // kV given (rwmg.cpp:641)
            c.cs = b.real("ctf.Cs");
            c.ast_angle = b.real("ctf.astigmatism_angle") * M_PI / 180.0;
            c.btx = b.real("ctf.beam_tilt_x");
            c.bty = b.real("ctf.beam_tilt_y");
        }
        const StarLoop* lp = b.loop_with("particle.id");
        const size_t n = lp ? lp->rows.size() : 0;
        auto col = [&](const char* tag, double def) {
            std::vector<double> v(n, def);
            const int i = lp ? lp->index(tag) : -1;
            if (i >= 0)
                for (size_t r = 0; r < n; ++r) v[r] = strtod(lp->rows[r][i].c_str(), nullptr);
            return v;
        };
        auto ids = col("particle.id", 0);
        mg.ox = col("particle.origin_x", 0);
        mg.oy = col("particle.origin_y", 0);
        auto oz = col("particle.origin_z", 0);
        if (lp && lp->index("particle.view_angle") >= 0) {
            mg.vx = col("particle.view_x", 0); mg.vy = col("particle.view_y", 0); mg.vz = col("particle.view_z", 1);
            mg.va = col("particle.view_angle", 0);
            for (auto& a : mg.va) a *= M_PI / 180.0;
        } else if (lp && (lp->index("particle.psi") >= 0 || lp->index("particle.omega") >= 0)) {
            // Euler (ZYZ) -> view (Euler.h:62-66)
            const bool psi = lp->index("particle.psi") >= 0;
            auto p = col(psi ? "particle.psi" : "particle.omega", 0);
            auto th = col("particle.theta", 0), ph = col("particle.phi", 0);
            for (size_t r = 0; r < n; ++r) {
                const double ps = (psi ? p[r] : -p[r]) * M_PI / 180.0, t = th[r] * M_PI / 180.0,
                             f = ph[r] * M_PI / 180.0;
                mg.vx.push_back(std::cos(f) * std::sin(t));
                mg.vy.push_back(std::sin(f) * std::sin(t));
                mg.vz.push_back(std::cos(t));
                mg.va.push_back(angle_neg_pi_to_pi(ps + f));
            }
        } else {
            mg.vx.assign(n, 0); mg.vy.assign(n, 0); mg.vz.assign(n, 1); mg.va.assign(n, 0);
        }
        mg.pixel = (lp && lp->index("particle.pixel_size_x") >= 0) ? col("particle.pixel_size_x", 0)
                                                                     : col("particle.pixel_size", 0);
        for (auto& p : mg.pixel)
            if (!(p > 0)) p = mg.pixel_size;
        mg.pixel_y = (lp && lp->index("particle.pixel_size_y") >= 0) ? col("particle.pixel_size_y", 0) : mg.pixel;
        for (size_t r = 0; r < mg.pixel_y.size(); ++r)
            if (!(mg.pixel_y[r] > 0)) mg.pixel_y[r] = mg.pixel[r];
        // read_project post-processing (rwmg.cpp:650-659): an origin further
        // than box_x/4 from the box centre (integer halves, z included) is
        // reset to the centre; then origin z = 0
        const double half[3] = {(double)(bs[0] / 2), (double)(bs[1] / 2), (double)(bs[2] / 2)};
        for (size_t r = 0; r < n; ++r) {
            const double d0 = mg.ox[r] - half[0], d1 = mg.oy[r] - half[1], d2 = oz[r] - half[2];
            if (std::sqrt(d0 * d0 + d1 * d1 + d2 * d2) > (double)(bs[0] / 4)) {
                mg.ox[r] = half[0];
                mg.oy[r] = half[1];
            }
        }
        mg.defocus = col("particle.defocus", 0);
        mg.mag = col("particle.magnification", 0);
        auto sel = col("particle.select", 1);
        for (size_t r = 0; r < n; ++r) {
            mg.part_id.push_back((long)ids[r]);
            mg.select.push_back((long)sel[r]);
        }
        out.push_back(std::move(mg));
    }
    if (out.empty()) throw std::runtime_error(path + ": no micrograph blocks found");
    return out;
}

// Point-group operators as rotation matrices (row-major, identity first) in
// the order of symmetry_get_all_views (bsoft/src/util/symmetry.cpp:277-319),
// from the generating operations of Bsymmetry::Bsymmetry (:42-115) and the
// label rules of clean_symstring (bsoft/include/symmetry.h:73-99): Cn, Dn,
// T, O, I and their -2/-3/-4/-5 variants.  Helical and I90 are rejected.
struct SymOp { double a[3]; int order; };

// The generating operations (axis as written, order) of Bsymmetry.
inline std::vector<SymOp> symmetry_generators(const std::string& sym) {
    std::string lbl;
    for (char ch : sym)
        if (!isspace((unsigned char)ch)) lbl += ch;
    if (lbl.empty()) lbl = "C1";
    if (isdigit((unsigned char)lbl[0])) {
        const int j = atoi(lbl.c_str());
        if (lbl.find("532") != std::string::npos) lbl = lbl.find("90") != std::string::npos ? "I90" : "I";
        else if (lbl.find("432") != std::string::npos) lbl = "O";
        else if (lbl.find("23") != std::string::npos) lbl = "T";
        else if (j > 1 && lbl.size() > 1 && lbl[1] == '2') lbl = "D" + std::to_string(j);
        else if (j > 0) lbl = "C" + std::to_string(j);
        else lbl = "C1";
    }
    lbl[0] = (char)toupper((unsigned char)lbl[0]);
    auto has = [&](const char* t) { return lbl.find(t) != std::string::npos; };
    const double gold = 1.61803398874989484820458683436563811772;
    using Op = SymOp;
    std::vector<Op> ops;
    if (lbl[0] == 'C') ops.push_back({{0, 0, 1}, lbl == "Cs" ? 1 : std::max(1, atoi(lbl.c_str() + 1))});
    else if (lbl[0] == 'D') { ops.push_back({{0, 0, 1}, atoi(lbl.c_str() + 1)}); ops.push_back({{1, 0, 0}, 2}); }
    else if (lbl[0] == 'T') {
        if (!has("-3")) ops.push_back({{1, 1, 1}, 3});
        ops.push_back({{0, 0, 1}, 2});
        ops.push_back({{1, 0, 0}, 2});
    } else if (lbl[0] == 'O') {
        if (!has("-3")) ops.push_back({{1, 1, 1}, 3});
        if (has("-4")) ops.push_back({{1, -1, 0}, 2});
        else if (has("-2")) ops.push_back({{0, 0, 1}, 4});
        else { ops.push_back({{0, 0, 1}, 4}); ops.push_back({{1, 0, 0}, 2}); }
    } else if (lbl[0] == 'I' && !has("90")) {
        if (!has("-3")) ops.push_back({{1, 1, 1}, 3});
        if (has("-5")) ops.push_back({{1, 0, 0}, 2});
        else if (has("-2")) ops.push_back({{1, -1, 0}, 2});
        else ops.push_back({{1, 1.0 / gold, gold}, 2});
        if (!has("-5")) ops.push_back({{1.0 / gold, 1, 0}, 5});
        if (!has("-2")) ops.push_back({{0, 0, 1}, 2});
    } else {
        throw std::runtime_error("unsupported symmetry " + sym);
    }
    return ops;
}

inline std::vector<double> symmetry_operators(const std::string& sym) {
    const std::vector<SymOp> ops = symmetry_generators(sym);
    std::vector<std::array<double, 4>> q{{1, 0, 0, 0}};
    for (const SymOp& op : ops) {
        const double n = std::sqrt(op.a[0] * op.a[0] + op.a[1] * op.a[1] + op.a[2] * op.a[2]);
        const size_t nv = q.size();
        for (int j = 1; j < op.order; ++j) {
            const double ang = j * 2.0 * M_PI / op.order, s = std::sin(ang / 2);
            const std::array<double, 4> g{std::cos(ang / 2), op.a[0] / n * s, op.a[1] / n * s, op.a[2] / n * s};
            for (size_t k = 0; k < nv; ++k) {
                const auto& p = q[k];
                q.push_back({g[0] * p[0] - g[1] * p[1] - g[2] * p[2] - g[3] * p[3],
                             g[0] * p[1] + g[1] * p[0] + g[2] * p[3] - g[3] * p[2],
                             g[0] * p[2] + g[2] * p[0] + g[3] * p[1] - g[1] * p[3],
                             g[0] * p[3] + g[3] * p[0] + g[1] * p[2] - g[2] * p[1]});
            }
        }
    }
    std::vector<double> m;
    for (const auto& t : q) {
        const double q0 = t[0], q1 = t[1], q2 = t[2], q3 = t[3];
        const double r[9] = {q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3, 2 * q1 * q2 - 2 * q0 * q3, 2 * q1 * q3 + 2 * q0 * q2,
                             2 * q1 * q2 + 2 * q0 * q3, q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3, 2 * q2 * q3 - 2 * q0 * q1,
                             2 * q1 * q3 - 2 * q0 * q2, 2 * q2 * q3 + 2 * q0 * q1, q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3};
        m.insert(m.end(), r, r + 9);
    }
    return m;
}

// The reference's View (x, y, z, angle) with its normalisation (View.h:30-35,
// 110-116: unit vector, components below 1e-30 zeroed, angle wrapped to
// [-pi, pi] and zeroed below 1e-30)
struct RefView {
    double v[3] = {0, 0, 1}, a = 0;
    void normalize() {
        const double size = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (size < TRIG) { v[0] = v[1] = 0; v[2] = 1; }
        else { v[0] /= size; v[1] /= size; v[2] /= size; }
        for (double& c : v)
            if (std::fabs(c) < TRIG) c = 0;
        a = angle_neg_pi_to_pi(a);
        if (std::fabs(a) < TRIG) a = 0;
    }
};

// symmetry_get_all_views (bsoft/src/util/symmetry.cpp:277-319): the view
// (copied by value, assigned, normalised), then for each generating
// operation and j = 1 .. order - 1, for each view so far, the quaternion of
// the rotation by j 2 pi / order about the operation's axis times the view's
// quaternion (View::quaternion, which normalises the stored view first),
// turned back into a View (View(Quaternion&), View.h:60-72).  Quaternion
// copies zero components below 1e-30 (Quaternion.h:28-32, 52-54).
inline std::vector<RefView> symmetry_views(const std::string& sym, double x, double y, double z, double a) {
    auto qcheck = [](double* q) {
        for (int i = 0; i < 4; ++i)
            if (std::fabs(q[i]) < TRIG) q[i] = 0;
    };
    auto view_quat = [&](RefView& w, double* q) {
        w.normalize();
        const double ang = (double)((long double)w.a / 2.0L);
        const double ca = std::cos(ang), sa = std::sin(ang);
        const double z1 = w.v[2] + 1;
        q[0] = ca; q[1] = 0; q[2] = 0; q[3] = sa;
        if (w.v[2] < 1.0L - TRIG) {
            if (w.v[2] <= TRIG - 1.0L) {
                q[0] = 0; q[1] = sa; q[2] = ca; q[3] = 0;
            } else {
                const double f1 = std::sqrt(z1 / 2.0), f2 = std::sqrt(1.0 / (2 * z1));
                q[0] = f1 * ca;
                q[1] = f2 * (w.v[0] * sa - w.v[1] * ca);
                q[2] = f2 * (w.v[0] * ca + w.v[1] * sa);
                q[3] = f1 * sa;
            }
        }
        qcheck(q);                                   // returned by value
    };
    RefView first;
    first.v[0] = x; first.v[1] = y; first.v[2] = z; first.a = a;
    first.normalize();                               // the by-value parameter
    first.normalize();                               // vn->normalize()
    std::vector<RefView> views{first};
    for (const SymOp& g : symmetry_generators(sym)) {
        // Bsymmetry stores the axis normalised; from_axis_angle normalises it again
        double ax[3] = {g.a[0], g.a[1], g.a[2]};
        for (int pass = 0; pass < 2; ++pass) {
            const double len = std::sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
            if (len < TRIG) { ax[0] = ax[1] = 0; ax[2] = 1; }
            else { const double d = 1.0 / len; ax[0] *= d; ax[1] *= d; ax[2] *= d; }
        }
        const size_t nv = views.size();
        for (int j = 1; j < g.order; ++j) {
            const double angle = (double)((long double)(j * 6.28318530717958647692528676655900576) / g.order);
            const double h = (double)((long double)angle / 2.0L);
            double q[4] = {std::cos(h), ax[0] * std::sin(h), ax[1] * std::sin(h), ax[2] * std::sin(h)};
            qcheck(q);
            for (size_t k = 0; k < nv; ++k) {
                double p[4];
                view_quat(views[k], p);
                double r[4];
                r[0] = q[0] * p[0] - (q[1] * p[1] + q[2] * p[2] + q[3] * p[3]);
                r[1] = q[0] * p[1] + q[1] * p[0] + q[2] * p[3] - q[3] * p[2];
                r[2] = q[0] * p[2] + q[2] * p[0] + q[3] * p[1] - q[1] * p[3];
                r[3] = q[0] * p[3] + q[3] * p[0] + q[1] * p[2] - q[2] * p[1];
                qcheck(r);                           // the product returned by value
                // View(Quaternion&)
                double ang = std::atan2(r[3], r[0]);
                const double ca = std::cos(ang), sa = std::sin(ang);
                const double q2 = r[0] * r[0] + r[3] * r[3];
                const double f2 = 2 * std::sqrt(q2);
                if (q2 < TRIG) ang = std::atan2(r[1], r[2]);
                RefView w;
                w.v[0] = f2 * (r[2] * ca + r[1] * sa);
                w.v[1] = f2 * (r[2] * sa - r[1] * ca);
                w.v[2] = 2 * q2 - 1;
                w.a = 2 * ang;
                w.normalize();
                views.push_back(w);
            }
        }
    }
    return views;
}

// STAR project with the particle parameters the readers above take, plus
// the figures of merit (mg_tags.h:227-228); one block per micrograph
inline void write_project(const std::string& path, const std::vector<Micrograph>& mgs,
                          const std::vector<std::vector<double>>& fom = {},
                          const std::vector<std::vector<double>>& fom_cv = {}) {
    const std::string tmp = path + ".tmp";
    FILE* f = fopen(tmp.c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + path);
    fprintf(f, "# Written by bsoft_b200\n\n");
    for (size_t m = 0; m < mgs.size(); ++m) {
        const Micrograph& mg = mgs[m];
        fprintf(f, "data_%s\n\n", mg.id.c_str());
        fprintf(f, "_micrograph.id %s\n_micrograph.pixel_size %.17g\n", mg.id.c_str(), mg.pixel_size);
        fprintf(f, "_particle.file_name '%s'\n", mg.particle_file.c_str());
        fprintf(f, "_particle.box_size_x %d\n_particle.box_size_y %d\n_particle.box_size_z 1\n", mg.box, mg.box);
        if (mg.has_ctf) {
            const Ctf& c = mg.ctf;
            fprintf(f, "_ctf.voltage %.17g\n_ctf.Cs %.17g\n_ctf.amplitude_phase_shift %.17g\n", c.volt, c.cs,
                    c.amp_shift);
            fprintf(f, "_ctf.defocus_average %.17g\n_ctf.defocus_deviation %.17g\n", c.defocus, c.def_dev);
            fprintf(f, "_ctf.astigmatism_angle %.17g\n", c.ast_angle * 180.0 / M_PI);
        }
        const bool has_fom = m < fom.size() && !fom[m].empty();
        fprintf(f, "\nloop_\n_particle.id\n_particle.defocus\n_particle.magnification\n_particle.pixel_size_x\n"
                   "_particle.pixel_size_y\n"
                   "_particle.origin_x\n_particle.origin_y\n_particle.origin_z\n_particle.view_x\n_particle.view_y\n"
                   "_particle.view_z\n_particle.view_angle\n_particle.select\n");
        if (has_fom) fprintf(f, "_particle.fom\n_particle.fom_crossvalidation\n");
        for (size_t i = 0; i < mg.part_id.size(); ++i) {
            const double py = i < mg.pixel_y.size() ? mg.pixel_y[i] : mg.pixel[i];
            fprintf(f, "%ld %.17g %.17g %.17g %.17g %.17g %.17g 0 %.17g %.17g %.17g %.17g %ld", mg.part_id[i],
                    mg.defocus[i], mg.mag[i], mg.pixel[i], py, mg.ox[i], mg.oy[i], mg.vx[i], mg.vy[i], mg.vz[i],
                    mg.va[i] * 180.0 / M_PI, mg.select[i]);
            if (has_fom) fprintf(f, " %.17g %.17g", fom[m][i], fom_cv[m][i]);
            fprintf(f, "\n");
        }
        fprintf(f, "\n");
    }
    if (fclose(f) != 0 || rename(tmp.c_str(), path.c_str()) != 0) throw std::runtime_error("cannot write " + path);
}

}  // namespace bsh
