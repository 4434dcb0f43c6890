// pf3d_ckpt.h -- binary checkpoint file of one domain (host side).
//
// The reference's only restart is its Tecplot snapshot read back as text
// (saida.f90:20-54 writes 8 significant digits; entrada.f90:284-321 reads
// them), which loses bits.  A checkpoint keeps the exact state of a domain so
// that a run continued from it gives the same bits as the run never stopped:
//
//   header (little-endian, 128 bytes)
//     char   magic[8]  = "PF3DCKP1"
//     int32  precision (64 | 32), nx, ny, nz, nfields (= 4)
//     int32  reserved
//     double dx, dy, dz
//     int64  it
//     double TP, M0, Cs_eq, Cl_eq
//     float  time, 4 bytes pad
//     uint64 deck hash (FNV-1a 64 over the deck values the step reads;
//            0 in files written before it was recorded: not checked)
//     pad to 128 bytes
//   4 fields in Fortran order without row padding, 8-byte doubles (precision
//   64) or 4-byte floats (precision 32): phase_field_old, conc_soluto_old,
//   TOLD, DPP -- the state every later step reads (the fused and the
//   per-subroutine steps overwrite every element of the "new" fields before
//   reading them).
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include "../../include/pf3d.h"

namespace pf3d {

struct CkptHeader {
    char magic[8];
    int32_t precision, nx, ny, nz, nfields, reserved;
    double dx, dy, dz;
    int64_t it;
    double TP, M0, Cs_eq, Cl_eq;
    float time;
    int32_t pad0;
    uint64_t deck_hash;
    char pad[128 - 8 - 6 * 4 - 3 * 8 - 8 - 4 * 8 - 4 - 4 - 8];
};
static_assert(sizeof(CkptHeader) == 128, "checkpoint header is 128 bytes");

constexpr int kCkptFields[4] = {PF_PHASE_OLD, PF_CONC_OLD, PF_TOLD, PF_DPP};

// FNV-1a 64 over the bytes of every deck value a continued run reads (the
// physics, the TP line and its cooling rate, the sweep count, h and noise
// forms); M0 (carried by the checkpoint's state) and the driver-only stop
// time and output cadence are left out.  Field by field, so struct padding
// never enters the hash.  Never 0.
inline uint64_t ckpt_deck_hash(const pf_params& p)
{
    uint64_t h = 0xcbf29ce484222325ull;
    auto mix = [&h](const void* v, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(v);
        for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 0x100000001b3ull;
    };
    const double d[] = {p.Tm, p.T0, p.delta_H, p.Cp_s, p.D, p.AAA, p.DELTA_EPSLON, p.D_sol, p.D_liq, p.Me,
                        p.Vm, p.R, p.C0, p.Thin_Interface, p.TP, p.taxa_resfr};
    const float f[] = {p.Ke, p.Sigma, p.Beta, p.ajuste};
    const int i[] = {p.n_varreduras, p.h_quintico, p.ruido_tipo, p.bc};
    mix(d, sizeof(d));
    mix(f, sizeof(f));
    mix(i, sizeof(i));
    return h ? h : 1;
}

inline CkptHeader ckpt_header(const pf_grid& g, int prec, const pf_state& st, const pf_params& p)
{
    CkptHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, "PF3DCKP1", 8);
    h.precision = prec;
    h.nx = g.nx;
    h.ny = g.ny;
    h.nz = g.nz;
    h.nfields = 4;
    h.dx = g.dx;
    h.dy = g.dy;
    h.dz = g.dz;
    h.it = st.it;
    h.TP = st.TP;
    h.M0 = st.M0;
    h.Cs_eq = st.Cs_eq;
    h.Cl_eq = st.Cl_eq;
    h.time = st.time;
    h.deck_hash = ckpt_deck_hash(p);
    return h;
}

inline pf_state ckpt_state(const CkptHeader& h)
{
    pf_state st{};
    st.it = (int)h.it;
    st.TP = h.TP;
    st.M0 = h.M0;
    st.Cs_eq = h.Cs_eq;
    st.Cl_eq = h.Cl_eq;
    st.time = h.time;
    return st;
}

// writes header + 4 fields of `field_bytes` each from `data`; "" on success
inline std::string ckpt_write(const std::string& path, const CkptHeader& h, const void* data, size_t field_bytes)
{
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return "cannot open " + path + " for writing";
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    if (ok && field_bytes) ok = std::fwrite(data, field_bytes, 4, f) == 4;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? std::string() : "short write to " + path;
}

// reads the header; checks magic, field count and that the grid (cells and
// spacing), the precision and the deck are the expected ones; "" on success
inline std::string ckpt_read_header(std::FILE* f, const pf_grid& g, int prec, const pf_params& p, CkptHeader* h)
{
    if (std::fread(h, sizeof(*h), 1, f) != 1) return "checkpoint shorter than its header";
    if (std::memcmp(h->magic, "PF3DCKP1", 8) != 0) return "not a checkpoint file";
    if (h->nfields != 4) return "unsupported field count";
    if (h->precision != prec) return "checkpoint precision differs from the domain's";
    if (h->nx != g.nx || h->ny != g.ny || h->nz != g.nz) return "checkpoint grid differs from the domain's";
    if (h->dx != g.dx || h->dy != g.dy || h->dz != g.dz) return "checkpoint grid spacing differs from the domain's";
    if (h->deck_hash != 0 && h->deck_hash != ckpt_deck_hash(p)) return "checkpoint deck differs from the domain's";
    return std::string();
}

}  // namespace pf3d
