// pf_karma3d.cpp -- the reference's Karma program (karma/karma3d.f90) on top
// of the C-ABI of include/pf3d.h.
//
//   pf_karma3d [--dir DIR] [--fp32] [--no-output] [--max-steps N]
//
// Reads DIR/karma.nml (the &karma namelist, karma3d.f90:80-113; defaults for
// names it does not set, the program's defaults when the file is absent),
// prints the run header of :126-137, seeds an eighth of a sphere at the
// corner on the device (:130-144) and runs the loop of :157-300: nout steps
// at a time on the GPU, then the tip line (largest i with phi > 0 on the x
// axis and on the diagonal), the Tecplot POINT file DIR/output/karma_<it>.dat
// of escreve (:341-359) and the stop test tip_x > tip_stop * N.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include <sys/stat.h>
#include "../../include/pf3d.h"
#include "pf_fortfmt.h"

namespace {

struct Run {
    pf_karma_params p{};
    long long nsteps = 100000, nout = 2000;
    double tip_stop = 0.9;
};

// karma3d.f90:80-92
void defaults(Run& r)
{
    pf_karma_params& p = r.p;
    p.nx = p.ny = p.nz = 200;
    p.lambda = 4.0;
    p.eps4 = 0.02;
    p.dx = 0.8;
    p.dt = 0.008;
    p.R0 = 8.0;
    p.Fnoise = 0.0;
    p.k = 0.14;
    p.Tm = 933.3;
    p.mliq = 640.0;
    p.C0 = 0.0196;
    p.TP = 909.5;
    p.sigma = 0.093;
    p.dH = 0.891002e9;
    p.Dl = 3.0e-9;
}

std::string lower(std::string s)
{
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// the &karma group of a namelist file: name = value pairs, '!' comments,
// commas or newlines between pairs, '/' ends the group
bool read_nml(const std::string& path, Run& r, std::string& err)
{
    std::ifstream f(path);
    if (!f) return true;   // karma3d.f90:104-110: no file, defaults
    std::stringstream ss;
    ss << f.rdbuf();
    std::string text = ss.str(), body;
    const size_t a = lower(text).find("&karma");
    if (a == std::string::npos) {
        err = "no &karma group";
        return false;
    }
    bool in_comment = false;
    for (size_t q = a + 6; q < text.size(); ++q) {
        const char c = text[q];
        if (c == '\n') in_comment = false;
        if (c == '!') in_comment = true;
        if (in_comment) continue;
        if (c == '/') break;
        body += (c == '\n') ? ',' : c;
    }
    std::map<std::string, double> v;
    std::stringstream items(body);
    std::string item;
    while (std::getline(items, item, ',')) {
        const size_t eq = item.find('=');
        if (eq == std::string::npos) continue;
        std::string key = item.substr(0, eq), val = item.substr(eq + 1);
        key.erase(std::remove_if(key.begin(), key.end(), ::isspace), key.end());
        for (char& c : val)
            if (c == 'd' || c == 'D') c = 'e';
        char* end = nullptr;
        const double x = std::strtod(val.c_str(), &end);
        if (end == val.c_str()) {
            err = "bad value for " + key;
            return false;
        }
        v[lower(key)] = x;
    }
    pf_karma_params& p = r.p;
    auto get = [&](const char* name, double& dst) {
        auto it = v.find(name);
        if (it != v.end()) dst = it->second;
    };
    if (v.count("n")) p.nx = p.ny = p.nz = (int)v["n"];
    get("lambda", p.lambda);
    get("eps4", p.eps4);
    get("dx", p.dx);
    get("dt", p.dt);
    get("r0", p.R0);
    get("fnoise", p.Fnoise);
    get("k", p.k);
    get("tm", p.Tm);
    get("mliq", p.mliq);
    get("c0", p.C0);
    get("tp", p.TP);
    get("sigma", p.sigma);
    get("dh", p.dH);
    get("dl", p.Dl);
    get("tip_stop", r.tip_stop);
    if (v.count("nsteps")) r.nsteps = (long long)v["nsteps"];
    if (v.count("nout")) r.nout = (long long)v["nout"];
    return true;
}

// escreve, karma3d.f90:341-359
bool escreve(const std::string& name, const pf_karma_params& p, const pf_karma_derived& dv,
             const std::vector<double>& phi, const std::vector<double>& U)
{
    FILE* f = std::fopen(name.c_str(), "w");
    if (!f) return false;
    std::fprintf(f, "TITLE=\"Phase Field (Karma)\"\n");
    std::fprintf(f, "variables= \"X\",\"Y\",\"Z\",\"PhaseField\",\"Temp\",\"Conc_Solute\"\n");
    std::fprintf(f, "ZONE\n");
    std::fprintf(f, " T=\" \" ,I= %d,J= %d,K= %d,F=POINT\n", p.nx, p.ny, p.nz);
    for (int c = 0; c < p.nz; ++c)
        for (int b = 0; b < p.ny; ++b)
            for (int a = 0; a < p.nx; ++a) {
                const size_t q = (size_t)a + (size_t)p.nx * ((size_t)b + (size_t)p.ny * c);
                const double cc = dv.cl0 * 0.5 * (1.0 + p.k - (1.0 - p.k) * phi[q]) * (1.0 + (1.0 - p.k) * U[q]);
                std::fprintf(f, " %s %s %s %s %s %s\n", fort_es15_7e3(a * p.dx * dv.W).c_str(),
                             fort_es15_7e3(b * p.dx * dv.W).c_str(), fort_es15_7e3(c * p.dx * dv.W).c_str(),
                             fort_es15_7e3(0.5 * (1.0 + phi[q])).c_str(), fort_es15_7e3(p.TP).c_str(),
                             fort_es15_7e3(cc).c_str());
            }
    std::fclose(f);
    return true;
}

int fail(const char* what, int rc)
{
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, pf_last_error(nullptr));
    return 1;
}

#define CALL(x, what)                          \
    do {                                       \
        int rc_ = (x);                         \
        if (rc_ != PF_OK) return fail(what, rc_); \
    } while (0)

}  // namespace

int main(int argc, char** argv)
{
    std::string dir = ".";
    bool fp32 = false, output = true;
    long long max_steps = -1;
    for (int a = 1; a < argc; ++a) {
        if (!std::strcmp(argv[a], "--dir") && a + 1 < argc) dir = argv[++a];
        else if (!std::strcmp(argv[a], "--fp32")) fp32 = true;
        else if (!std::strcmp(argv[a], "--no-output")) output = false;
        else if (!std::strcmp(argv[a], "--max-steps") && a + 1 < argc) max_steps = std::atoll(argv[++a]);
        else {
            std::fprintf(stderr, "usage: pf_karma3d [--dir DIR] [--fp32] [--no-output] [--max-steps N]\n");
            return 2;
        }
    }
    Run r;
    defaults(r);
    std::string err;
    if (!read_nml(dir + "/karma.nml", r, err)) {
        std::fprintf(stderr, "erro lendo karma.nml: %s\n", err.c_str());
        return 1;
    }
    if (max_steps >= 0) r.nsteps = std::min(r.nsteps, max_steps);
    const pf_karma_params& p = r.p;
    pf_karma_derived dv{};
    CALL(pf_karma_derived_of(&p, &dv), "pf_karma_derived_of");
    const int N = p.nx;

    // karma3d.f90:126-137
    std::printf("### karma3d -- campo de fase quantitativo (Karma 2001 / EFKP 2004) ###\n");
    std::printf("N = %d^3,  dx = %6.3f W,  dominio = %8.3f um\n", N, p.dx, N * p.dx * dv.W * 1.0e6);
    std::printf("k = %6.3f  eps4 = %6.3f  lambda = %6.3f  D = %7.3f\n", p.k, p.eps4, p.lambda, dv.D);
    std::printf("TP = %8.2f K   c_l0 = %8.5f   Omega = %6.3f\n", p.TP, dv.cl0, dv.Omega);
    std::printf("d0 = %s m   W = %s m   tau0 = %s s\n", fort_es(dv.d0, 10, 3).c_str(), fort_es(dv.W, 10, 3).c_str(),
                fort_es(dv.tau0, 10, 3).c_str());
    std::printf("dt = %s s   (%lld passos max)   Fnoise = %7.4f\n", fort_es(p.dt * dv.tau0, 10, 3).c_str(), r.nsteps,
                p.Fnoise);
    if (dv.D * p.dt / (p.dx * p.dx) > 0.3 / 3.0 || p.dt / (p.dx * p.dx) > 0.4 / 3.0)
        std::printf("AVISO: dt perto do limite de estabilidade explicita\n");
    std::printf("### GPU (B200, %s) ###\n", fp32 ? "FP32" : "FP64");
    std::fflush(stdout);

    pf_karma* k = nullptr;
    CALL(pf_karma_create(&p, fp32 ? PF_FP32 : PF_FP64, &k), "pf_karma_create");
    CALL(pf_karma_seed(k), "pf_karma_seed");
    if (output) mkdir((dir + "/output").c_str(), 0755);
    const size_t cells = (size_t)p.nx * p.ny * p.nz;
    std::vector<double> phi, U;
    const auto t0 = std::chrono::steady_clock::now();
    long long it = 0;
    while (it < r.nsteps) {
        // the next output event: mod(it, nout) == 0 or it == nsteps
        const long long next = std::min(r.nsteps, (it / r.nout + 1) * r.nout);
        CALL(pf_karma_step(k, (int)(next - it)), "pf_karma_step");
        it = next;
        int tip_x = 0, tip_d = 0;
        CALL(pf_karma_tip(k, &tip_x, &tip_d), "pf_karma_tip");
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        const double s3 = std::sqrt(3.0);
        std::printf("it=%8lld  t=%10.1f tau0 (%s s)  ponta_eixo=%7.1f W  ponta_diag=%7.1f W  razao=%6.3f  wall=%8.1f s\n",
                    it, it * p.dt, fort_es(it * p.dt * dv.tau0, 10, 3).c_str(), tip_x * p.dx, tip_d * p.dx * s3,
                    tip_x / std::max(tip_d * s3, 1.0), wall);
        std::fflush(stdout);
        if (output) {
            phi.resize(cells);
            U.resize(cells);
            CALL(pf_karma_download(k, PF_KARMA_PHI, phi.data()), "pf_karma_download");
            CALL(pf_karma_download(k, PF_KARMA_U, U.data()), "pf_karma_download");
            char name[64];
            std::snprintf(name, sizeof name, "/output/karma_%07lld.dat", it);
            if (!escreve(dir + name, p, dv, phi, U)) std::fprintf(stderr, "escreve: cannot write %s\n", name);
        }
        if (tip_x > r.tip_stop * N) {
            std::printf("### ponta chegou perto da parede -- fim ###\n");
            break;
        }
    }
    pf_karma_destroy(k);
    return 0;
}
