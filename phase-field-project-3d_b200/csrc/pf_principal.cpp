// pf_principal.cpp -- the reference's main program (source/principal.f90) on
// top of the C-ABI of include/pf3d.h.
//
//   pf_principal [--dir DIR] [--fused] [--quiet] [--max-steps N] [--no-output]
//
// Reads DIR/entrada.dat like entrada.f90 (three header lines, then the first
// value of each line, optional trailing lines with their defaults), builds
// the initial state of entrada.f90:226-262 (tipo_inicial 0-3) or reads
// DIR/restart.dat (tipo_inicial 4, with the k_desl shift of :284-321), and
// runs the time loop of principal.f90:93-259:
//   temperatura -> TP ramp -> n_varreduras phase sweeps (copy between) ->
//   concentracao_soluto -> auxiliar -> [output event] -> swap -> stop test,
// each subroutine a C-ABI call.  With --fused the steps between output
// events run as pf_step (same results).  Output events follow the E_R
// counter (first at it = WriteFileD_timeCounter + 1): the diagnostics line,
// and the Tecplot POINT file of saida.f90 in DIR/output/ (formatted and
// written by a host thread while the loop steps on).  The progress line
// of equacao_campo_fase.f90:174 is printed per sweep unless --quiet.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include <thread>
#include <sys/stat.h>
#include "../../include/pf3d.h"
#include "pf_fortfmt.h"

namespace {

struct Deck {
    pf_grid g{};
    pf_params p{};
    long long it_max = 0;
    int tipo_inicial = 0;
    double R_semente = 0.0;
};


bool first_values(const std::string& line, int n, double* out)
{
    std::istringstream is(line);
    for (int q = 0; q < n; ++q) {
        std::string tok;
        if (!(is >> tok)) return false;
        char* end = nullptr;
        std::string t = tok;
        for (char& ch : t)
            if (ch == 'd' || ch == 'D') ch = 'e';
        out[q] = std::strtod(t.c_str(), &end);
        if (end == t.c_str()) return false;
    }
    return true;
}

// entrada.f90:17-89
bool read_deck(const std::string& path, Deck& d, std::string& err)
{
    std::ifstream f(path);
    if (!f) { err = "cannot open " + path; return false; }
    std::vector<std::string> L;
    std::string s;
    while (std::getline(f, s)) L.push_back(s);
    if (L.size() < 3 + 36) { err = "entrada.dat too short"; return false; }
    auto v = [&](int k) { double x = 0; if (!first_values(L[3 + k], 1, &x)) x = 0; return x; };
    pf_params& p = d.p;
    std::memset(&p, 0, sizeof(p));
    p.Tm = v(0); p.T0 = v(1); p.delta_H = v(2); p.M0 = v(5); p.Cp_s = v(8);
    d.g.nx = (int)v(10); d.g.ny = (int)v(11); d.g.nz = (int)v(12);
    d.g.dy = v(13); d.g.dx = v(14); d.g.dz = v(15);
    d.it_max = (long long)v(18);
    p.AAA = v(19);
    p.DELTA_EPSLON = v(21);
    p.D_sol = v(23); p.D_liq = v(24);
    p.Ke = (float)v(25);
    p.Me = v(26); p.Vm = v(27); p.R = v(28); p.C0 = v(29); p.Thin_Interface = v(30);
    p.Sigma = (float)v(31); p.Beta = (float)v(32); p.ajuste = (float)v(33);
    p.stoptime = v(34);
    p.WriteFileD_timeCounter = (int)v(35);
    double a[2];
    // optional lines (iostat defaults)
    p.TP = (L.size() > 3 + 36 && first_values(L[3 + 36], 1, a)) ? a[0] : 919.0;
    if (L.size() > 3 + 37 && first_values(L[3 + 37], 2, a)) { d.tipo_inicial = (int)a[0]; d.R_semente = a[1]; }
    if (L.size() > 3 + 38 && first_values(L[3 + 38], 2, a)) { p.taxa_resfr = a[0]; p.n_varreduras = (int)a[1]; }
    else { p.taxa_resfr = 0.0; p.n_varreduras = 1; }
    if (p.n_varreduras < 1) p.n_varreduras = 1;
    if (L.size() > 3 + 39 && first_values(L[3 + 39], 2, a)) { p.h_quintico = (int)a[0]; p.ruido_tipo = (int)a[1]; }
    else { p.h_quintico = 1; p.ruido_tipo = 2; }
    p.D = 0.0;   // the reference's module variable D is never assigned
    p.bc = PF_BC_REFERENCE;
    return true;
}

size_t at(const pf_grid& g, int i, int j, int k)
{
    return (size_t)(i - 1) + (size_t)g.nx * ((size_t)(j - 1) + (size_t)g.ny * (size_t)(k - 1));
}

// entrada.f90:226-262
void init_fields(const Deck& d, std::vector<double>& phi, std::vector<double>& c, std::vector<double>& T)
{
    const pf_grid& g = d.g;
    int ic = g.nx / 2, jc = g.ny / 2, kc = g.nz / 2;
    if (d.tipo_inicial == 2) ic = jc = kc = 3;
    const double Ke = (double)d.p.Ke;
    for (int k = 1; k <= g.nz; ++k)
        for (int j = 1; j <= g.ny; ++j)
            for (int i = 1; i <= g.nx; ++i) {
                double dist2 = 1.7976931348623157e308;
                if (d.tipo_inicial == 1 || d.tipo_inicial == 2)
                    dist2 = (double)(i - ic) * (i - ic) + (double)(j - jc) * (j - jc) + (double)(k - kc) * (k - kc);
                const bool solid = (d.tipo_inicial == 0 && j <= 4) || (d.tipo_inicial == 3 && k <= 4) ||
                                   dist2 <= d.R_semente * d.R_semente;
                const size_t q = at(g, i, j, k);
                phi[q] = solid ? 1.0 : 0.0;
                c[q] = solid ? Ke * d.p.C0 : d.p.C0;
                T[q] = d.p.T0;
            }
}

// entrada.f90:284-321 (restart.dat: 4 header lines, then X Y Z phi T c per cell)
bool read_restart(const std::string& path, const Deck& d, std::vector<double>& phi, std::vector<double>& c,
                  std::string& err)
{
    const pf_grid& g = d.g;
    const int kd = std::max(0, (int)std::lround(d.R_semente));
    if (kd >= g.nz) { err = "tipo_inicial = 4: deslocamento >= Nz"; return false; }
    std::ifstream f(path);
    if (!f) { err = "tipo_inicial = 4: restart.dat nao encontrado"; return false; }
    std::string s;
    for (int q = 0; q < 4; ++q) std::getline(f, s);
    for (int kk = 1; kk <= g.nz; ++kk)
        for (int jj = 1; jj <= g.ny; ++jj)
            for (int ii = 1; ii <= g.nx; ++ii) {
                double x, y, z, ph, t, cr;
                if (!(f >> x >> y >> z >> ph >> t >> cr)) { err = "tipo_inicial = 4: restart.dat menor que a malha"; return false; }
                const int kn = kk - kd;
                if (kn >= 1) {
                    phi[at(g, ii, jj, kn)] = ph;
                    c[at(g, ii, jj, kn)] = cr;
                }
                if (kk == g.nz && kd > 0)
                    for (int k2 = g.nz - kd + 1; k2 <= g.nz; ++k2) {
                        phi[at(g, ii, jj, k2)] = 0.0;
                        c[at(g, ii, jj, k2)] = cr;
                    }
            }
    return true;
}

// saida.f90:20-54
bool saida(const std::string& dir, const pf_grid& g, int it, float time, double TP, const std::vector<double>& phi,
           const std::vector<double>& c)
{
    char text[16], text2[32];
    std::snprintf(text, sizeof text, "%6d", it);
    std::snprintf(text2, sizeof text2, "%14.7f", (double)time);
    auto rtrim = [](std::string v) { while (!v.empty() && v.back() == ' ') v.pop_back(); return v; };
    std::string name = "saida_" + rtrim(text) + "_time_" + rtrim(text2) + "s.dat";
    std::string path = dir + "/output/" + name;
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    std::fprintf(f, " TITLE=\"Phase Field\"\n");
    std::fprintf(f, "variables= \"X\",\"Y\",\"Z\",\"PhaseField\",\"Temp\",\"Conc_Solute\"\n");
    std::fprintf(f, " ZONE\n");
    std::fprintf(f, " T=\" \" ,I=%4d,J=%4d,K=%4d,F=POINT\n", g.nx, g.ny, g.nz);
    for (int k = 1; k <= g.nz; ++k)
        for (int j = 1; j <= g.ny; ++j)
            for (int i = 1; i <= g.nx; ++i) {
                const size_t q = at(g, i, j, k);
                std::fprintf(f, " %s %s %s %s %s %s\n", fort_es15_7e3((i - 1) * g.dx).c_str(),
                             fort_es15_7e3((j - 1) * g.dy).c_str(), fort_es15_7e3((k - 1) * g.dz).c_str(),
                             fort_es15_7e3(phi[q]).c_str(), fort_es15_7e3(TP).c_str(), fort_es15_7e3(c[q]).c_str());
            }
    std::fprintf(f, "        \n        \n");
    std::fclose(f);
    return true;
}

// Tecplot output off the time loop: the fields of an output event are copied
// to the host, and a writer thread formats and writes them while the loop
// steps on (one file in flight; the next event waits for it).
class SaidaWriter {
public:
    SaidaWriter(std::string dir, pf_grid g) : dir_(std::move(dir)), g_(g) {}
    ~SaidaWriter() { wait(); }
    // takes the buffers (swapped out of the caller's vectors)
    void submit(int it, float time, double TP, std::vector<double>& phi, std::vector<double>& c)
    {
        wait();
        phi_.swap(phi);
        c_.swap(c);
        th_ = std::thread([this, it, time, TP]() {
            if (!saida(dir_, g_, it, time, TP, phi_, c_)) ok_ = false;
        });
    }
    void wait()
    {
        if (th_.joinable()) th_.join();
    }
    bool ok() const { return ok_; }

private:
    std::string dir_;
    pf_grid g_;
    std::vector<double> phi_, c_;
    std::thread th_;
    bool ok_ = true;
};

int fail(const char* what, pf_ctx* ctx, int rc)
{
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, pf_last_error(ctx));
    return 1;
}

#define CALL(x, what)                                  \
    do {                                               \
        int rc_ = (x);                                 \
        if (rc_ != PF_OK) return fail(what, ctx, rc_); \
    } while (0)

}  // namespace

int main(int argc, char** argv)
{
    std::string dir = ".";
    bool fused = false, quiet = false, output = true;
    long long max_steps = -1;
    for (int a = 1; a < argc; ++a) {
        std::string s = argv[a];
        if (s == "--dir" && a + 1 < argc) dir = argv[++a];
        else if (s == "--fused") fused = true;
        else if (s == "--quiet") quiet = true;
        else if (s == "--no-output") output = false;
        else if (s == "--max-steps" && a + 1 < argc) max_steps = std::atoll(argv[++a]);
        else {
            std::fprintf(stderr, "usage: pf_principal [--dir DIR] [--fused] [--quiet] [--no-output] [--max-steps N]\n");
            return 2;
        }
    }
    Deck d;
    std::string err;
    if (!read_deck(dir + "/entrada.dat", d, err)) { std::fprintf(stderr, "%s\n", err.c_str()); return 1; }
    const pf_grid& g = d.g;
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    std::vector<double> phi(n), c(n), T(n), dpp(n, 0.0);
    init_fields(d, phi, c, T);
    if (d.tipo_inicial == 4 && !read_restart(dir + "/restart.dat", d, phi, c, err)) {
        std::fprintf(stderr, "%s\n", err.c_str());
        return 1;
    }
    pf_ctx* ctx = nullptr;
    CALL(pf_create(&g, &d.p, PF_FP64, &ctx), "pf_create");
    pf_derived dv;
    pf_get_derived(ctx, &dv);
    std::printf(" W0==> %.15E      E0==> %.15E      Dt==> %.15E\n", dv.W0, dv.E0, dv.DELTA_T);   // W0_E0.f90:33
    // target enter data (principal.f90:60-64)
    CALL(pf_upload(ctx, PF_PHASE_OLD, phi.data()), "upload phase_field_old");
    CALL(pf_upload(ctx, PF_CONC_OLD, c.data()), "upload conc_soluto_old");
    CALL(pf_upload(ctx, PF_TOLD, T.data()), "upload TOLD");
    CALL(pf_upload(ctx, PF_DPP, dpp.data()), "upload DPP");
    if (output) mkdir((dir + "/output").c_str(), 0755);
    SaidaWriter writer(dir, g);

    pf_state st;
    pf_get_state(ctx, &st);
    double TP = st.TP, M0 = st.M0, Cs_eq = 0, Cl_eq = 0;
    float time = 0.0f;
    const int counter = d.p.WriteFileD_timeCounter;
    int E_R = 0;   // the reference leaves it uninitialised; static storage starts at 0
    const long long last = max_steps >= 0 ? std::min(d.it_max, max_steps) : d.it_max;
    const auto t0 = std::chrono::steady_clock::now();
    for (long long it = 1; it <= last; ++it) {
        const float time_prev = time;
        time = (float)(dv.DELTA_T + (double)time);                              // :96
        const bool out_now = counter > 0 && E_R >= counter;
        if (fused && !out_now && quiet) {
            // one fused step; the context advances it, time, TP and M0 itself
            pf_state s2{(int)it - 1, TP, M0, Cs_eq, Cl_eq, time_prev};
            pf_set_state(ctx, &s2);
            CALL(pf_step(ctx, 1), "pf_step");
            pf_get_state(ctx, &s2);
            TP = s2.TP; M0 = s2.M0; Cs_eq = s2.Cs_eq; Cl_eq = s2.Cl_eq; time = s2.time;
        } else {
            CALL(pf_temperatura(ctx, TP), "temperatura");                       // :98
            if (d.p.taxa_resfr > 0.0) TP = d.p.T0 - d.p.taxa_resfr * dv.DELTA_T * (double)it;   // :104
            for (int sw = 1; sw <= d.p.n_varreduras; ++sw) {                     // :127-152
                if (sw > 1) CALL(pf_copy_phase_new_to_old(ctx), "copy phase");
                CALL(pf_equacao_campo_fase(ctx, (int)it, TP, M0, &Cs_eq, &Cl_eq), "equacao_campo_fase");
                if (!quiet) {
                    double p1, p2;
                    CALL(pf_probe(ctx, PF_PHASE_NEW, g.nx / 2, 10, std::max(g.nz / 2, 1), &p1), "probe");
                    CALL(pf_probe(ctx, PF_PHASE_NEW, g.nx / 2, std::min(100, g.ny - 1), std::max(g.nz / 2, 1), &p2), "probe");
                    std::printf(" %s %s %s\n", fort_e(p1, 14, 4).c_str(), fort_e(TP, 14, 4).c_str(), fort_e(p2, 14, 4).c_str());
                }
            }
            CALL(pf_concentracao_soluto(ctx), "concentracao_soluto");           // :154
            CALL(pf_auxiliar(ctx, TP, Cs_eq, Cl_eq, &M0), "auxiliar");           // :157
            if (out_now) {                                                       // :161-186
                E_R = 0;
                std::printf("=====================================================\n");
                std::printf("=============  ESCREVENDO RESULTADOS  ===============\n");
                std::printf("IT==> %8lld iteracoes\n", it);
                double dg[5];
                CALL(pf_diagnosticos(ctx, dg), "diagnosticos");
                std::printf("L2(phi)==>%s  phi_max==>%s  phi_min==>%s  solute_total==>%s  free_energy==>%s\n",
                            fort_e(dg[0], 14, 6).c_str(), fort_e(dg[1], 14, 6).c_str(), fort_e(dg[2], 14, 6).c_str(),
                            fort_e(dg[3], 14, 6).c_str(), fort_e(dg[4], 14, 6).c_str());
                if (output) {
                    phi.resize(n);
                    c.resize(n);
                    CALL(pf_download(ctx, PF_PHASE_NEW, phi.data()), "download phase_field_new");
                    CALL(pf_download(ctx, PF_CONC_NEW, c.data()), "download conc_soluto_new");
                    writer.submit((int)it, time, TP, phi, c);
                }
            }
            CALL(pf_swap(ctx), "swap");                                          // :200-226
            pf_state s2{(int)it, TP, M0, Cs_eq, Cl_eq, time};
            pf_set_state(ctx, &s2);
        }
        E_R = E_R + 1;                                                           // :187
        if (d.p.stoptime != 0.0 && (double)time >= d.p.stoptime) {               // :233-254
            std::printf("     Program terminated by stop time condition = %14.7f s\n", d.p.stoptime);
            break;
        }
    }
    CALL(pf_sync(ctx), "sync");
    writer.wait();
    if (!writer.ok()) std::fprintf(stderr, "saida: cannot write\n");
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    pf_get_state(ctx, &st);
    std::printf("Average Time/Step      : %.5f s\n", secs / std::max(1, st.it));
    // final state for a caller that inspects it: old fields after the swap
    if (output) {
        phi.resize(n);
        c.resize(n);
        CALL(pf_download(ctx, PF_PHASE_OLD, phi.data()), "download");
        CALL(pf_download(ctx, PF_CONC_OLD, c.data()), "download");
        FILE* f = std::fopen((dir + "/output/final_state.bin").c_str(), "wb");
        if (f) {
            std::fwrite(phi.data(), sizeof(double), n, f);
            std::fwrite(c.data(), sizeof(double), n, f);
            std::fclose(f);
        }
    }
    pf_destroy(ctx);
    return 0;
}
