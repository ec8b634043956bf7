// common.h -- shared pieces of the drop-in programs AFor, AVSPRTM and decon2d_mine.
//
// parameter.txt is a sequence of (label line, value) pairs read with fgets + fscanf exactly
// as the reference does (acoustic_HLVSPRTMC.cpp:1931-2035, forward/...HLForC.cpp:2059-2163,
// kk_decon_interp_psf_minewindow.cpp:1527-1629), so any file the reference accepts parses
// identically.  After the pairs the reference stops reading; lines of the form
// `swd.key = value` anywhere after them are this project's extensions (device, strip
// precision, scatter perturbation type) and are ignored by the reference.
#pragma once
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <string>
#include <vector>
#include <map>
#include <initializer_list>
#include "swd.h"

namespace drv {

struct ParamReader {
    FILE *fp = nullptr;
    char line[256];
    bool ok = true;
    explicit ParamReader(const char *path) { fp = fopen(path, "r"); }
    ~ParamReader()
    {
        if (fp) fclose(fp);
    }
    void label()
    {
        if (!fgets(line, 256, fp)) ok = false;
        if (fscanf(fp, "\n") < 0) ok = false;
    }
    void get(int *v) { label(); if (fscanf(fp, "%d", v) != 1) ok = false; if (fscanf(fp, "\n") < 0) {} }
    void get(float *v) { label(); if (fscanf(fp, "%f", v) != 1) ok = false; if (fscanf(fp, "\n") < 0) {} }
    void get(char *s) { label(); if (fscanf(fp, "%149s", s) != 1) ok = false; if (fscanf(fp, "\n") < 0) {} }
};

// `swd.key = value` extension lines anywhere in the file
inline std::map<std::string, std::string> extensions(const char *path)
{
    std::map<std::string, std::string> kv;
    FILE *fp = fopen(path, "r");
    if (!fp) return kv;
    char buf[512];
    while (fgets(buf, sizeof buf, fp)) {
        char *p = buf;
        while (*p == ' ' || *p == '\t') p++;
        if (strncmp(p, "swd.", 4) != 0) continue;
        char *eq = strchr(p, '=');
        if (!eq) continue;
        std::string k(p + 4, eq - p - 4), v(eq + 1);
        auto trim = [](std::string &s) {
            size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
            s = a == std::string::npos ? "" : s.substr(a, b - a + 1);
        };
        trim(k);
        trim(v);
        kv[k] = v;
    }
    fclose(fp);
    return kv;
}

inline int ext_int(const std::map<std::string, std::string> &kv, const char *k, int def)
{
    auto it = kv.find(k);
    return it == kv.end() ? def : atoi(it->second.c_str());
}
inline float ext_float(const std::map<std::string, std::string> &kv, const char *k, float def)
{
    auto it = kv.find(k);
    return it == kv.end() ? def : (float)atof(it->second.c_str());
}
inline std::string ext_str(const std::map<std::string, std::string> &kv, const char *k, const char *def)
{
    auto it = kv.find(k);
    return it == kv.end() ? std::string(def) : it->second;
}
// An extension whose value must be one of `choices` (the first is the default).  An unknown
// value is reported and the caller stops before any device work, instead of running with a
// silent default.
inline bool ext_choice(const std::map<std::string, std::string> &kv, const char *k,
                       std::initializer_list<const char *> choices, std::string &out)
{
    auto it = kv.find(k);
    out = it == kv.end() ? std::string(*choices.begin()) : it->second;
    std::string all;
    for (const char *c : choices) {
        if (out == c) return true;
        all += (all.empty() ? "" : "|") + std::string(c);
    }
    printf("swd.%s = %s: expected %s\n", k, out.c_str(), all.c_str());
    return false;
}

inline bool write_f32(const std::string &path, const float *a, size_t n)
{
    FILE *fp = fopen(path.c_str(), "wb");
    if (!fp) {
        fprintf(stderr, "Cannot write the file: %s\n", path.c_str());
        return false;
    }
    size_t w = fwrite(a, sizeof(float), n, fp);
    fclose(fp);
    return w == n;
}

inline bool read_f32(const std::string &path, float *a, size_t n)
{
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp) {
        printf("Cannot Open the File: %s\n", path.c_str());
        return false;
    }
    size_t r = fread(a, sizeof(float), n, fp);
    fclose(fp);
    if (r != n) {
        printf("The file %s holds %zu of the %zu floats expected\n", path.c_str(), r, n);
        return false;
    }
    return true;
}

// interior (nx x nz) view of a padded (ntx x ntz) grid, in file order (x-major, z fastest)
inline std::vector<float> interior(const std::vector<float> &g, int ntx, int ntz, int pmlc)
{
    std::vector<float> out;
    out.reserve((size_t)(ntx - 2 * pmlc) * (ntz - 2 * pmlc));
    for (int ix = pmlc; ix <= ntx - pmlc - 1; ix++)
        for (int iz = pmlc; iz <= ntz - pmlc - 1; iz++) out.push_back(g[(size_t)ix * ntz + iz]);
    return out;
}

inline void die_on(swd_ctx *ctx, int rc, const char *what)
{
    if (rc != SWD_OK) {
        fprintf(stderr, "%s failed (%d): %s\n", what, rc, swd_last_error(ctx));
        exit(1);
    }
}

// Modelling/RTM parameters, acoustic_HLVSPRTMC.cpp:1931-2035 (18 pairs)
struct ModelParams {
    int nx, nz, pml, Lc, itmax, ns, scatter_flag, swin, window;
    float dx, dz, dt, f0, sx0, shotdx, shotdep, recdix, offsetz;
};

inline bool read_model_params(const char *path, ModelParams &m)
{
    ParamReader r(path);
    if (!r.fp) return false;
    r.get(&m.nx); r.get(&m.nz); r.get(&m.pml); r.get(&m.Lc); r.get(&m.dx); r.get(&m.dz);
    r.get(&m.itmax); r.get(&m.dt); r.get(&m.f0); r.get(&m.ns); r.get(&m.sx0); r.get(&m.shotdx);
    r.get(&m.shotdep); r.get(&m.recdix); r.get(&m.offsetz); r.get(&m.scatter_flag); r.get(&m.swin);
    r.get(&m.window);
    return r.ok;
}

// Size of a file in bytes, or -1 when it cannot be opened.
inline long long file_bytes(const std::string &path)
{
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp) return -1;
    fseek(fp, 0, SEEK_END);
    const long long n = ftell(fp);
    fclose(fp);
    return n;
}

// A seismogram record [r_n][itmax] (trace-major float32, the layout AFor writes): the file must
// hold exactly r_n * itmax floats.  The reference freads r_n*itmax floats without looking
// (acoustic_HLVSPRTMC.cpp:598-604), so a record of another receiver count or length would be
// migrated silently as garbage; here the mismatch is reported with both shapes.
inline bool check_record(const std::string &path, int r_n, int itmax)
{
    const long long n = file_bytes(path);
    if (n < 0) {
        printf("Cannot Open the File: %s\n", path.c_str());
        return false;
    }
    const long long want = (long long)r_n * itmax * (long long)sizeof(float);
    if (n != want) {
        printf("The file %s holds %lld floats; r_n x itmax = %d x %d = %lld expected\n", path.c_str(),
               n / (long long)sizeof(float), r_n, itmax, want / (long long)sizeof(float));
        return false;
    }
    return true;
}

// Receivers of shot `is` (0-based).  The optional file <root>/input/<is+1>source_receivers.txt
// gives the shot its own receiver list: the count r_n, then r_n lines "ix iz" of interior cell
// indices (0 <= ix < nx, 0 <= iz < nz).  Without it the shot has the reference's two edge wells
// (acoustic_HLVSPRTMC.cpp:153-200), the same for every shot.  Returns false, with a message,
// for a malformed file.
struct Receivers {
    std::vector<int> ix, iz;   // padded-grid cells
    bool from_file = false;
};

inline bool shot_receivers(const std::string &root, int is, const ModelParams &m, Receivers &R)
{
    const int pmlc = m.pml + m.Lc;
    char name[256];
    snprintf(name, sizeof name, "%s/input/%dsource_receivers.txt", root.c_str(), is + 1);
    FILE *fp = fopen(name, "r");
    R.ix.clear();
    R.iz.clear();
    R.from_file = fp != nullptr;
    if (!fp) {
        const int r_n = swd_prep_wells(m.nx, m.nz, pmlc, m.dz, m.shotdep, m.offsetz, nullptr, nullptr);
        if (r_n < 2) {
            printf("No receiver depth lies within the maximum offset\n");
            return false;
        }
        R.ix.resize(r_n);
        R.iz.resize(r_n);
        swd_prep_wells(m.nx, m.nz, pmlc, m.dz, m.shotdep, m.offsetz, R.ix.data(), R.iz.data());
        return true;
    }
    int r_n = 0;
    bool ok = fscanf(fp, "%d", &r_n) == 1 && r_n >= 1;
    for (int k = 0; ok && k < r_n; k++) {
        int x, z;
        if (fscanf(fp, "%d %d", &x, &z) != 2) {
            printf("%s: %d receivers announced, %d read\n", name, r_n, k);
            ok = false;
            break;
        }
        if (x < 0 || x >= m.nx || z < 0 || z >= m.nz) {
            printf("%s: receiver %d at (%d, %d) lies outside the %d x %d model\n", name, k, x, z, m.nx, m.nz);
            ok = false;
            break;
        }
        R.ix.push_back(pmlc + x);
        R.iz.push_back(pmlc + z);
    }
    if (!ok && R.ix.empty() && r_n < 1) printf("%s: no receiver count\n", name);
    fclose(fp);
    return ok;
}

// Stencil coefficients, CPML profiles and stability print shared by AFor and AVSPRTM
// (acoustic_HLVSPRTMC.cpp:106-118, 462-469).
struct Operator {
    std::vector<float> rc, ax, axh, az, azh, bx, bxh, bz, bzh;
};

inline Operator make_operator(const ModelParams &m, int ntx, int ntz, int pmlc)
{
    Operator o;
    o.rc.resize(m.Lc);
    swd_prep_xishu(m.Lc, o.rc.data());
    float tmprc = 0.0;
    for (int ic = 0; ic < m.Lc; ic++) tmprc += fabsf(o.rc[ic]);
    printf("Maximum velocity for stability is %f m/s\n", m.dx / (tmprc * m.dt * sqrt(2)));
    o.ax.resize(ntx); o.axh.resize(ntx); o.bx.resize(ntx); o.bxh.resize(ntx);
    o.az.resize(ntz); o.azh.resize(ntz); o.bz.resize(ntz); o.bzh.resize(ntz);
    swd_prep_cpml(ntx, ntz, pmlc, m.dx, m.dz, m.dt, o.ax.data(), o.axh.data(), o.az.data(), o.azh.data(),
                  o.bx.data(), o.bxh.data(), o.bz.data(), o.bzh.data());
    return o;
}

inline swd_ctx *make_context(const ModelParams &m, int device)
{
    swd_grid g{m.nx, m.nz, m.pml, m.Lc, m.dx, m.dz, m.dt, m.itmax, device};
    swd_ctx *ctx = nullptr;
    int rc = swd_create(&ctx, &g);
    if (rc != SWD_OK) {
        fprintf(stderr, "swd_create failed (%d): no usable CUDA device or invalid grid\n", rc);
        exit(1);
    }
    return ctx;
}

}  // namespace drv
