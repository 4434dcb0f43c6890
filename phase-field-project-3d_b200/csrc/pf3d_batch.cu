// pf3d_batch.cu -- many independent domains stepped together (C-ABI pf_batch_*).
//
// A batch holds up to max_domains domains of one precision, each with its own
// grid, deck and step count, under a device-memory budget.  All active
// domains advance together: one persistent kernel per pass walks a work list
// of (domain, tile) items, and K steps are captured once in a CUDA graph.
// Everything that changes between launches lives in device tables the host
// rewrites in stream order:
//   doms   : descriptor and buffer pointers of every slot,
//   items  : the work list (rebuilt when membership or the tile shape changes),
//   steps  : per step and slot the step scalars (TP, M0, it, ...), whether the
//            slot advances in that step, and which buffer holds the old field.
// So domains join and leave between graph launches without recapture
// (continuous batching), and a slot that reaches its target step count stops
// while the others go on.  Per-domain results are the same bits as stepping
// that domain alone: the tile function is the one of pf_step and no value
// depends on the tile shape, the z-chunk or the other domains.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>
#include "../../include/pf3d.h"
#include "pf3d_hostdesc.h"
#include "pf3d_ckpt.h"
#include "pf3d_init.cuh"
#include "pf3d_tma.cuh"
#include "pf3d_tmap.h"

using namespace pf3d;

namespace pf3d {
int set_last_error_global(int code, const std::string& msg);
}

namespace {

constexpr int kGraphSteps = 8;   // steps per captured graph

struct Slot {
    bool used = false;
    pf_grid g{};
    pf_params p{};
    pf_derived dv{};
    pf_state st{};
    long long target = 0;     // stop after this step (0 = no limit)
    int qphi = 0, qc = 0, qT = 0;
    void* mem = nullptr;
    size_t bytes = 0;
    BatchDomain bd{};
};

// autotuner cache: shape class -> (tile_y, zchunk)
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, std::tuple<int, int, int>> g_tune_cache;   // -> tile_y, zchunk, pair

}  // namespace

struct pf_batch {
    int prec = 64;
    size_t es = 8;
    long long budget = 0, used_bytes = 0;
    int max_domains = 0;
    int nsw = 0;                       // sweeps per step shared by all slots (1 or 2)
    std::vector<Slot> slots;
    BatchDomain* d_doms = nullptr;
    BatchStep* d_steps = nullptr;      // kGraphSteps x max_domains
    BatchStep* h_steps[2] = {nullptr, nullptr};
    cudaEvent_t h_ev[2] = {nullptr, nullptr};
    int h_cur = 0;
    BatchItem* d_items = nullptr;
    int item_cap = 0;
    int* d_nitems = nullptr;
    bool items_dirty = true;
    double* d_part = nullptr;          // diagnostics partials (592 x kDiagRow) + result
    unsigned long long* d_track = nullptr;   // tracking scratch (grown to the tallest slot tracked)
    int track_cap = 0;                 // planes it holds
    double* h_out = nullptr;
    double* d_sites = nullptr;         // bump sites for device initialisation
    int tile_y = 8, zchunk = 64, n_sm = 0;   // persistent grids: n_sm x resident CTAs
    int pair = 0;                      // 32 x 8 tiles with two cells per thread (set by the autotuner)
    int march = 1;                     // TMA-staged march passes (32 x 8 tiles); 0: the cp.async passes
    int nslot = 0;                     // window mode of the march passes (0: 3)
    CUtensorMap* d_tmaps = nullptr;    // 2 per slot: the tensor maps of its phase-field buffers
    int* d_ctr = nullptr;              // work-item counters of a graph's launches (2 per step)
    int* d_status = nullptr;           // kernel status word (0, or the code a kernel left there)
    cudaStream_t own_stream = nullptr, stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_ty = 0, graph_zc = 0, graph_nsm = 0, graph_nsw = 0, graph_march = -1, graph_nslot = 0;
    bool graph_smooth = false, graph_pair = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    bool pending = false;              // steps enqueued by pf_batch_step_async not yet waited for
    long long last_steps = 0;
    std::string err;
};

static int berr(pf_batch* b, int code, const std::string& msg)
{
    if (b) b->err = msg;
    return set_last_error_global(code, msg);
}

#define BCK(call, what)                                                                  \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) return berr(b, PF_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
    } while (0)

static bool b64(const pf_batch* b) { return b->prec == PF_FP64; }

static int rebuild_items(pf_batch* b)
{
    std::vector<BatchItem> items;
    // largest domains first: their items are the longest-running
    std::vector<int> order;
    for (int s = 0; s < (int)b->slots.size(); ++s)
        if (b->slots[s].used) order.push_back(s);
    std::sort(order.begin(), order.end(), [&](int a, int c) {
        const pf_grid& ga = b->slots[a].g;
        const pf_grid& gc = b->slots[c].g;
        return (long long)ga.nz > (long long)gc.nz || (ga.nz == gc.nz && a < c);
    });
    for (int s : order) {
        const pf_grid& g = b->slots[s].g;
        const int nbx = (g.nx + 31) / 32, nby = (g.ny + b->tile_y - 1) / b->tile_y;
        const int nbz = (g.nz + b->zchunk - 1) / b->zchunk;
        for (int bz = 0; bz < nbz; ++bz)
            for (int by = 0; by < nby; ++by)
                for (int bx = 0; bx < nbx; ++bx) items.push_back(BatchItem{s, bx, by, bz});
    }
    const int n = (int)items.size();
    if (n > b->item_cap) {
        BCK(cudaStreamSynchronize(b->stream), "work list resize");
        if (b->d_items) cudaFree(b->d_items);
        if (b->graph) {   // the captured launches point at the old list
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        b->item_cap = std::max(n, 2 * b->item_cap);
        BCK(cudaMalloc(&b->d_items, (size_t)b->item_cap * sizeof(BatchItem)), "work list");
    }
    if (n) BCK(cudaMemcpyAsync(b->d_items, items.data(), n * sizeof(BatchItem), cudaMemcpyHostToDevice, b->stream),
               "work list upload");
    BCK(cudaMemcpyAsync(b->d_nitems, &n, sizeof(int), cudaMemcpyHostToDevice, b->stream), "work list size");
    BCK(cudaStreamSynchronize(b->stream), "work list sync");   // the host vector goes out of scope
    b->items_dirty = false;
    return PF_OK;
}

// whether any domain of the batch draws the smooth noise (ruido_tipo 2): the
// first-pass kernels carry that code only when one does
static bool any_smooth(const pf_batch* b)
{
    for (const Slot& sl : b->slots)
        if (sl.used && sl.p.ruido_tipo == 2) return true;
    return false;
}

// whether any domain of the batch diffuses heat (D > 0)
static bool any_lap(const pf_batch* b)
{
    for (const Slot& sl : b->slots)
        if (sl.used && sl.p.D != 0.0) return true;
    return false;
}

static bool use_march(const pf_batch* b) { return b->march && b->tile_y == 8; }

static int capture_graph(pf_batch* b)
{
    const bool smooth = any_smooth(b);
    const bool march = use_march(b);
    const int nslot = b->nslot ? b->nslot : 3;
    // two cells per thread on 32 x 8 tiles when the autotuner measured it
    // faster: the march passes in either precision (not with the smooth
    // noise); the cp.async passes in FP32 only, on decks without heat
    // diffusion (their boundary tiles run the one-cell code twice)
    const bool pair = march ? (b->pair && !smooth)
                            : (b->pair && !b64(b) && b->tile_y == 8 && !smooth && !any_lap(b));
    if (b->graph && b->graph_ty == b->tile_y && b->graph_zc == b->zchunk && b->graph_nsm == b->n_sm &&
        b->graph_nsw == b->nsw && b->graph_smooth == smooth && b->graph_pair == pair &&
        b->graph_march == (int)march && b->graph_nslot == nslot)
        return PF_OK;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaStream_t cs;
    BCK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess && march)   // the work counters of the graph's launches start at zero
        e = cudaMemsetAsync(b->d_ctr, 0, 2 * kGraphSteps * sizeof(int), cs);
    if (e == cudaSuccess) {
        for (int k = 0; k < kGraphSteps && e == cudaSuccess; ++k) {
            const BatchStep* st = b->d_steps + (size_t)k * b->max_domains;
            const bool one = b->nsw == 1;
            if (march) {
                const int lanes = pair ? 2 : 1;
                for (int pass = 0; pass <= (one ? 0 : 1) && e == cudaSuccess; ++pass)
                    e = b64(b) ? launch_march_batch<double>(b->d_doms, b->d_tmaps, st, b->d_items, b->d_nitems, pass,
                                                            one, smooth && pass == 0, lanes, nslot, b->zchunk,
                                                            b->n_sm, b->d_ctr + 2 * k + pass, b->d_status, cs)
                               : launch_march_batch<float>(b->d_doms, b->d_tmaps, st, b->d_items, b->d_nitems, pass,
                                                           one, smooth && pass == 0, lanes, nslot, b->zchunk,
                                                           b->n_sm, b->d_ctr + 2 * k + pass, b->d_status, cs);
                continue;
            }
            if (pair) {
                e = launch_fused_batch_pair<float>(b->d_doms, st, b->d_items, b->d_nitems, 0, one, b->zchunk, b->n_sm,
                                                   cs);
                if (e == cudaSuccess && !one)
                    e = launch_fused_batch_pair<float>(b->d_doms, st, b->d_items, b->d_nitems, 1, false, b->zchunk,
                                                       b->n_sm, cs);
                continue;
            }
            e = b64(b) ? launch_fused_batch<double>(b->d_doms, st, b->d_items, b->d_nitems, 0, one, smooth, b->tile_y,
                                                    b->zchunk, b->n_sm, cs)
                       : launch_fused_batch<float>(b->d_doms, st, b->d_items, b->d_nitems, 0, one, smooth, b->tile_y,
                                                   b->zchunk, b->n_sm, cs);
            if (e == cudaSuccess && !one)
                e = b64(b) ? launch_fused_batch<double>(b->d_doms, st, b->d_items, b->d_nitems, 1, false, false,
                                                        b->tile_y, b->zchunk, b->n_sm, cs)
                           : launch_fused_batch<float>(b->d_doms, st, b->d_items, b->d_nitems, 1, false, false,
                                                       b->tile_y, b->zchunk, b->n_sm, cs);
        }
        cudaError_t e2 = cudaStreamEndCapture(cs, &g);
        if (e == cudaSuccess) e = e2;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) return berr(b, PF_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    b->graph_ty = b->tile_y;
    b->graph_zc = b->zchunk;
    b->graph_nsm = b->n_sm;
    b->graph_nsw = b->nsw;
    b->graph_smooth = smooth;
    b->graph_pair = pair;
    b->graph_march = (int)march;
    b->graph_nslot = nslot;
    return PF_OK;
}

static int set_grid(pf_batch* b)
{
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    b->n_sm = std::max(1, nsm);
    return PF_OK;
}

// Fills step table rows for up to kGraphSteps steps; returns how many steps
// any slot advances.  Advances each slot's host state like pf_step does.
static int fill_steps(pf_batch* b, BatchStep* rows, int nsteps)
{
    int advanced = 0;
    std::memset(rows, 0, sizeof(BatchStep) * (size_t)kGraphSteps * b->max_domains);
    for (int k = 0; k < kGraphSteps; ++k) {
        for (int sidx = 0; sidx < (int)b->slots.size(); ++sidx) {
            Slot& sl = b->slots[sidx];
            BatchStep& r = rows[(size_t)k * b->max_domains + sidx];
            r.active = 0;
            if (!sl.used || k >= nsteps) continue;
            if (sl.target > 0 && sl.st.it >= sl.target) continue;
            const pf_params& p = sl.p;
            const int it = sl.st.it + 1;
            const double dt = sl.dv.DELTA_T;
            const double TP_heat = sl.st.TP;
            const double TP = step_tp(p, dt, it, sl.st.TP);
            r.s = make_step_args(p, sl.dv, it, TP_heat, TP, sl.st.M0);
            if (b->prec == PF_FP64) {
                KC<double> kc;
                kc.load(sl.bd.d, r.s);
                std::memcpy(r.kc, &kc, sizeof(kc));
            } else {
                KC<float> kc;
                kc.load(sl.bd.d, r.s);
                std::memcpy(r.kc, &kc, sizeof(kc));
            }
            r.active = 1;
            r.q_phi = sl.qphi;
            r.q_c = sl.qc;
            r.q_T = sl.qT;
            // host state after the step (principal.f90:96-157 and the swap)
            sl.st.time = (float)(dt + (double)sl.st.time);
            if (b->nsw == 1) sl.qphi ^= 1;   // the new phase lands in the other buffer
            sl.qc ^= 1;
            sl.qT ^= 1;
            double Cs, Cl, M0n;
            equilibrium(p, TP, &Cs, &Cl);
            pf_auxiliar_scalar(&p, sl.dv.E0, sl.dv.W0, TP, Cs, Cl, &M0n);
            sl.st.M0 = M0n;
            sl.st.TP = TP;
            sl.st.Cs_eq = Cs;
            sl.st.Cl_eq = Cl;
            sl.st.it = it;
            advanced = std::max(advanced, k + 1);
        }
    }
    return advanced;
}

extern "C" {

int pf_batch_create(int precision, long long budget_bytes, int max_domains, pf_batch** out)
{
    if (!out) return set_last_error_global(PF_E_ARG, "pf_batch_create: out is null");
    *out = nullptr;
    if ((precision != PF_FP64 && precision != PF_FP32) || max_domains < 1 || max_domains > 65536 || budget_bytes < 0)
        return set_last_error_global(PF_E_ARG, "pf_batch_create: bad precision, max_domains or budget");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_last_error_global(PF_E_NODEV, "no CUDA device visible");
    }
    pf_batch* b = new pf_batch();
    b->prec = precision;
    b->es = precision == PF_FP32 ? 4 : 8;
    b->budget = budget_bytes;
    b->max_domains = max_domains;
    b->slots.resize(max_domains);
    cudaError_t e = cudaSuccess;
    const size_t step_bytes = sizeof(BatchStep) * (size_t)kGraphSteps * max_domains;
    if ((e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_doms, sizeof(BatchDomain) * (size_t)max_domains)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_steps, step_bytes)) != cudaSuccess ||
        (e = cudaMallocHost(&b->h_steps[0], step_bytes)) != cudaSuccess ||
        (e = cudaMallocHost(&b->h_steps[1], step_bytes)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_nitems, sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_part, (592 * kDiagRow + 8) * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_sites, 2 * 4096 * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_tmaps, sizeof(CUtensorMap) * 2 * (size_t)max_domains)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_status, sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_ctr, 2 * kGraphSteps * sizeof(int))) != cudaSuccess ||
        (e = cudaMallocHost(&b->h_out, 8 * sizeof(double))) != cudaSuccess ||
        (e = cudaEventCreate(&b->h_ev[0])) != cudaSuccess || (e = cudaEventCreate(&b->h_ev[1])) != cudaSuccess ||
        (e = cudaEventCreate(&b->ev0)) != cudaSuccess || (e = cudaEventCreate(&b->ev1)) != cudaSuccess) {
        pf_batch_destroy(b);
        return set_last_error_global(PF_E_CUDA, std::string("pf_batch_create: ") + cudaGetErrorString(e));
    }
    b->stream = b->own_stream;
    // slots come from the device's stream-ordered pool (cudaMallocAsync):
    // adding and removing a domain then neither waits for the GPU nor stops
    // it; up to 8 GB of freed slot memory stays cached for the next ones
    {
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = 8ull << 30, cur = 0;
            if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur) == cudaSuccess && cur < keep)
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    }
    cudaMemset(b->d_steps, 0, step_bytes);
    cudaMemset(b->d_nitems, 0, sizeof(int));
    cudaMemset(b->d_status, 0, sizeof(int));
    if (!tmap_encoder()) b->march = 0;   // no tensor-map encoder in this driver: the cp.async passes
    set_grid(b);
    *out = b;
    return PF_OK;
}

int pf_batch_destroy(pf_batch* b)
{
    if (!b) return PF_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto& s : b->slots)
        if (s.mem) cudaFree(s.mem);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    cudaFree(b->d_doms);
    cudaFree(b->d_steps);
    cudaFreeHost(b->h_steps[0]);
    cudaFreeHost(b->h_steps[1]);
    cudaFree(b->d_items);
    cudaFree(b->d_nitems);
    cudaFree(b->d_part);
    if (b->d_track) cudaFree(b->d_track);
    cudaFree(b->d_sites);
    cudaFree(b->d_tmaps);
    cudaFree(b->d_status);
    cudaFree(b->d_ctr);
    cudaFreeHost(b->h_out);
    for (cudaEvent_t ev : {b->h_ev[0], b->h_ev[1], b->ev0, b->ev1})
        if (ev) cudaEventDestroy(ev);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    delete b;
    return PF_OK;
}

int pf_batch_set_stream(pf_batch* b, void* stream)
{
    if (!b) return PF_E_ARG;
    b->stream = stream ? (cudaStream_t)stream : b->own_stream;
    return PF_OK;
}

long long pf_batch_bytes_used(const pf_batch* b) { return b ? b->used_bytes : -1; }

int pf_batch_count(const pf_batch* b)
{
    if (!b) return -1;
    int n = 0;
    for (const auto& s : b->slots) n += s.used ? 1 : 0;
    return n;
}

int pf_batch_add(pf_batch* b, const pf_grid* g, const pf_params* p, int* slot)
{
    if (!b || !slot) return berr(b, PF_E_ARG, "pf_batch_add: bad argument");
    *slot = -1;
    std::string why;
    int rc = validate(g, p, b->prec, why);
    if (rc) return berr(b, rc, "pf_batch_add: " + why);
    if (p->n_varreduras > 2) return berr(b, PF_E_ARG, "pf_batch_add: batches support 1 or 2 sweeps per step");
    if (b->nsw != 0 && p->n_varreduras != b->nsw && pf_batch_count(b) > 0)
        return berr(b, PF_E_ARG, "pf_batch_add: every domain of a batch must use the same n_varreduras");
    int s = -1;
    for (int i = 0; i < (int)b->slots.size(); ++i)
        if (!b->slots[i].used) { s = i; break; }
    if (s < 0) return berr(b, PF_E_NOMEM, "pf_batch_add: all slots are in use");
    const int px = pitch_of(g->nx);
    const size_t fb = round_up((size_t)px * g->ny * g->nz * b->es + 64, 256);
    const size_t bytes = 7 * fb;
    if (b->budget > 0 && b->used_bytes + (long long)bytes > b->budget)
        return berr(b, PF_E_NOMEM, "pf_batch_add: over the device-memory budget");
    Slot& sl = b->slots[s];
    sl = Slot();
    void* mem = nullptr;
    cudaError_t e = cudaMallocAsync(&mem, bytes, b->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return berr(b, PF_E_NOMEM, std::string("pf_batch_add: cudaMallocAsync: ") + cudaGetErrorString(e));
    }
    cudaMemsetAsync(mem, 0, bytes, b->stream);
    sl.used = true;
    sl.g = *g;
    sl.p = *p;
    setup_derived(*g, *p, sl.dv);
    sl.st.it = 0;
    sl.st.TP = initial_tp(*p);
    sl.st.M0 = p->M0;
    sl.st.time = 0.0f;
    equilibrium(*p, sl.st.TP, &sl.st.Cs_eq, &sl.st.Cl_eq);
    sl.mem = mem;
    sl.bytes = bytes;
    fill_desc(*g, *p, sl.dv, px, sl.bd.d);
    char* m = (char*)mem;
    sl.bd.phi[0] = m;
    sl.bd.phi[1] = m + fb;
    sl.bd.c[0] = m + 2 * fb;
    sl.bd.c[1] = m + 3 * fb;
    sl.bd.T[0] = m + 4 * fb;
    sl.bd.T[1] = m + 5 * fb;
    sl.bd.dpp = m + 6 * fb;
    // from pageable memory: staged at the call, so no wait is needed
    BCK(cudaMemcpyAsync(b->d_doms + s, &sl.bd, sizeof(BatchDomain), cudaMemcpyHostToDevice, b->stream), "descriptor");
    if (b->march) {
        CUtensorMap tm[2];
        for (int q = 0; q < 2; ++q)
            if (encode_field_map(&tm[q], sl.bd.phi[q], (int)b->es, g->nx, g->ny, g->nz, px, march_box_x((int)b->es),
                                 march_box_y(8)) != 0) {
                cudaFreeAsync(mem, b->stream);
                sl = Slot();
                return berr(b, PF_E_CUDA, "pf_batch_add: tensor map encoding failed");
            }
        BCK(cudaMemcpyAsync(b->d_tmaps + 2 * (size_t)s, tm, sizeof(tm), cudaMemcpyHostToDevice, b->stream),
            "tensor maps");
    }
    b->used_bytes += (long long)bytes;
    b->nsw = p->n_varreduras;
    b->items_dirty = true;
    *slot = s;
    return PF_OK;
}

int pf_batch_remove(pf_batch* b, int slot)
{
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
        return berr(b, PF_E_ARG, "pf_batch_remove: bad slot");
    Slot& sl = b->slots[slot];
    // stream-ordered: released after the steps already queued that use it
    BCK(cudaFreeAsync(sl.mem, b->stream), "remove");
    b->used_bytes -= (long long)sl.bytes;
    sl = Slot();
    b->items_dirty = true;
    return PF_OK;
}

static void* slot_field(Slot& sl, int field)
{
    switch (field) {
    case PF_PHASE_OLD: return sl.bd.phi[sl.qphi];
    case PF_PHASE_NEW: return sl.bd.phi[1 - sl.qphi];
    case PF_CONC_OLD: return sl.bd.c[sl.qc];
    case PF_CONC_NEW: return sl.bd.c[1 - sl.qc];
    case PF_TOLD: return sl.bd.T[sl.qT];
    case PF_TNEW: return sl.bd.T[1 - sl.qT];
    case PF_DPP: return sl.bd.dpp;
    }
    return nullptr;
}

static Slot* get_slot(pf_batch* b, int slot)
{
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used) return nullptr;
    return &b->slots[slot];
}

int pf_batch_upload(pf_batch* b, int slot, int field, const double* host)
{
    Slot* sl = get_slot(b, slot);
    if (!sl || !host || field < 0 || field > 6) return berr(b, PF_E_ARG, "pf_batch_upload: bad argument");
    const pf_grid& g = sl->g;
    void* dst = slot_field(*sl, field);
    if (b64(b)) {
        BCK(cudaMemcpy2DAsync(dst, (size_t)sl->bd.d.px * 8, host, (size_t)g.nx * 8, (size_t)g.nx * 8,
                              (size_t)g.ny * g.nz, cudaMemcpyHostToDevice, b->stream),
            "pf_batch_upload");
    } else {
        // through the staging area of the diagnostics buffer is too small; use a temporary
        const size_t n = (size_t)g.nx * g.ny * g.nz;
        double* stage = nullptr;
        BCK(cudaMalloc(&stage, n * sizeof(double)), "pf_batch_upload staging");
        cudaError_t e = cudaMemcpyAsync(stage, host, n * sizeof(double), cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess) e = launch_convert_in<float>(sl->bd.d, stage, dst, 0, g.nz, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        cudaFree(stage);
        if (e != cudaSuccess) return berr(b, PF_E_CUDA, std::string("pf_batch_upload: ") + cudaGetErrorString(e));
    }
    BCK(cudaStreamSynchronize(b->stream), "pf_batch_upload sync");
    return PF_OK;
}

int pf_batch_download(pf_batch* b, int slot, int field, double* host)
{
    Slot* sl = get_slot(b, slot);
    if (!sl || !host || field < 0 || field > 6) return berr(b, PF_E_ARG, "pf_batch_download: bad argument");
    const pf_grid& g = sl->g;
    void* src = slot_field(*sl, field);
    if (b64(b)) {
        BCK(cudaMemcpy2DAsync(host, (size_t)g.nx * 8, src, (size_t)sl->bd.d.px * 8, (size_t)g.nx * 8,
                              (size_t)g.ny * g.nz, cudaMemcpyDeviceToHost, b->stream),
            "pf_batch_download");
    } else {
        const size_t n = (size_t)g.nx * g.ny * g.nz;
        double* stage = nullptr;
        BCK(cudaMalloc(&stage, n * sizeof(double)), "pf_batch_download staging");
        cudaError_t e = launch_convert_out<float>(sl->bd.d, src, stage, 0, g.nz, b->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(host, stage, n * sizeof(double), cudaMemcpyDeviceToHost, b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        cudaFree(stage);
        if (e != cudaSuccess) return berr(b, PF_E_CUDA, std::string("pf_batch_download: ") + cudaGetErrorString(e));
    }
    BCK(cudaStreamSynchronize(b->stream), "pf_batch_download sync");
    return PF_OK;
}

int pf_batch_init_seeded(pf_batch* b, int slot, int n_bumps, const double* sites)
{
    Slot* sl = get_slot(b, slot);
    if (!sl || n_bumps < 0 || n_bumps > 4096 || (n_bumps > 0 && !sites))
        return berr(b, PF_E_ARG, "pf_batch_init_seeded: bad argument (at most 4096 bumps)");
    InitArgs a;
    a.n_bumps = n_bumps;
    a.slab_top = 4.5;
    a.bump_r = 3.0;
    a.width = sl->p.Thin_Interface;
    a.kmax = std::min(sl->g.nz, (int)(a.slab_top + a.bump_r + 20.0 * a.width / 2.0) + 2);
    a.C0 = sl->p.C0;
    a.Ke = (double)sl->p.Ke;
    a.T0 = sl->p.T0;
    if (n_bumps)
        BCK(cudaMemcpyAsync(b->d_sites, sites, 2 * n_bumps * sizeof(double), cudaMemcpyHostToDevice, b->stream),
            "bump sites");
    cudaError_t e = b64(b) ? launch_init_seeded<double>(sl->bd.d, a, b->d_sites, slot_field(*sl, PF_PHASE_OLD),
                                                        slot_field(*sl, PF_CONC_OLD), slot_field(*sl, PF_TOLD),
                                                        sl->bd.dpp, b->stream)
                           : launch_init_seeded<float>(sl->bd.d, a, b->d_sites, slot_field(*sl, PF_PHASE_OLD),
                                                       slot_field(*sl, PF_CONC_OLD), slot_field(*sl, PF_TOLD),
                                                       sl->bd.dpp, b->stream);
    BCK(e, "pf_batch_init_seeded");
    BCK(cudaStreamSynchronize(b->stream), "pf_batch_init_seeded sync");
    return PF_OK;
}

int pf_batch_set_target(pf_batch* b, int slot, long long target_it)
{
    Slot* sl = get_slot(b, slot);
    if (!sl || target_it < 0) return berr(b, PF_E_ARG, "pf_batch_set_target: bad argument");
    sl->target = target_it;
    return PF_OK;
}

int pf_batch_get_state(const pf_batch* b, int slot, pf_state* out)
{
    if (!b || !out || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used) return PF_E_ARG;
    *out = b->slots[slot].st;
    return PF_OK;
}

int pf_batch_progress(const pf_batch* b, int* it, int n)
{
    if (!b || !it || n < 0) return PF_E_ARG;
    for (int s = 0; s < n; ++s)
        it[s] = (s < (int)b->slots.size() && b->slots[s].used) ? b->slots[s].st.it : -1;
    return PF_OK;
}

int pf_batch_set_paired(pf_batch* b, int paired)
{
    if (!b || paired < 0 || paired > 1) return berr(b, PF_E_ARG, "pf_batch_set_paired: 0 or 1");
    b->pair = paired;
    return PF_OK;
}

int pf_batch_set_kernel(pf_batch* b, int kernel, int nslot)
{
    if (!b || kernel < 0 || kernel > 1 || (nslot != 0 && nslot != 3 && nslot != 4 && nslot != 5))
        return berr(b, PF_E_ARG, "pf_batch_set_kernel: kernel 0 or 1, window mode 0, 3, 4 or 5");
    if (kernel == 1 && !tmap_encoder())
        return berr(b, PF_E_STATE, "pf_batch_set_kernel: this driver has no tensor-map encoder");
    if (kernel == 1 && !b->march) {
        // slots added while the march passes were off have no tensor maps yet
        for (int s = 0; s < (int)b->slots.size(); ++s) {
            Slot& sl = b->slots[s];
            if (!sl.used) continue;
            CUtensorMap tm[2];
            for (int q = 0; q < 2; ++q)
                if (encode_field_map(&tm[q], sl.bd.phi[q], (int)b->es, sl.g.nx, sl.g.ny, sl.g.nz, sl.bd.d.px,
                                     march_box_x((int)b->es), march_box_y(8)) != 0)
                    return berr(b, PF_E_CUDA, "pf_batch_set_kernel: tensor map encoding failed");
            BCK(cudaMemcpyAsync(b->d_tmaps + 2 * (size_t)s, tm, sizeof(tm), cudaMemcpyHostToDevice, b->stream),
                "tensor maps");
        }
    }
    b->march = kernel;
    b->nslot = nslot;
    return PF_OK;
}

int pf_batch_set_tile(pf_batch* b, int tile_y, int zchunk)
{
    if (!b || (tile_y != 4 && tile_y != 8 && tile_y != 16) || zchunk < 1)
        return berr(b, PF_E_ARG, "pf_batch_set_tile: tile_y in {4, 8, 16}, zchunk >= 1");
    if (tile_y != b->tile_y || zchunk != b->zchunk) {
        b->tile_y = tile_y;
        b->zchunk = zchunk;
        b->items_dirty = true;
        set_grid(b);
    }
    return PF_OK;
}

// Enqueues up to n_steps steps as graphs of kGraphSteps steps; the host fills
// the next step table while the GPU runs the current graph (two tables,
// reused after their upload has completed).  Returns without waiting.
int pf_batch_step_async(pf_batch* b, int n_steps)
{
    if (!b || n_steps < 0) return berr(b, PF_E_ARG, "pf_batch_step_async: bad argument");
    if (b->items_dirty) {
        int rc = rebuild_items(b);
        if (rc) return rc;
    }
    int rc = capture_graph(b);
    if (rc) return rc;
    long long steps_done = 0;
    int left = n_steps;
    bool launched = false;
    while (left > 0) {
        const int chunk = std::min(left, kGraphSteps);
        const int hb = b->h_cur;
        BCK(cudaEventSynchronize(b->h_ev[hb]), "step table reuse");
        const int adv = fill_steps(b, b->h_steps[hb], chunk);
        left -= chunk;
        if (adv == 0) break;   // every slot reached its target
        BCK(cudaMemcpyAsync(b->d_steps, b->h_steps[hb], sizeof(BatchStep) * (size_t)kGraphSteps * b->max_domains,
                            cudaMemcpyHostToDevice, b->stream),
            "step table upload");
        BCK(cudaEventRecord(b->h_ev[hb], b->stream), "step table event");
        b->h_cur ^= 1;
        if (!launched) BCK(cudaEventRecord(b->ev0, b->stream), "timing event");
        BCK(cudaGraphLaunch(b->graph, b->stream), "graph launch");
        launched = true;
        steps_done += adv;
    }
    if (launched) BCK(cudaEventRecord(b->ev1, b->stream), "timing event");
    b->pending = launched;
    b->last_ms = 0.0;
    b->last_steps = steps_done;
    return PF_OK;
}

// the kernel status word, after the stream has drained: PF_E_KERNEL when a
// kernel reported a failure (cleared once reported)
static int batch_status(pf_batch* b)
{
    int code = 0;
    BCK(cudaMemcpyAsync(&code, b->d_status, sizeof(int), cudaMemcpyDeviceToHost, b->stream), "status read");
    BCK(cudaStreamSynchronize(b->stream), "status read");
    if (code == 0) return PF_OK;
    BCK(cudaMemsetAsync(b->d_status, 0, sizeof(int), b->stream), "status reset");
    return berr(b, PF_E_KERNEL, "a batch kernel reported failure code " + std::to_string(code) +
                                    (code == kErrTmaTimeout ? " (a TMA plane load did not arrive in time)" : ""));
}

// Waits for the steps of the last pf_batch_step_async; their device time is
// then pf_batch_last_ms.
int pf_batch_wait(pf_batch* b)
{
    if (!b) return berr(b, PF_E_ARG, "pf_batch_wait: bad argument");
    if (!b->pending) return PF_OK;
    BCK(cudaEventSynchronize(b->ev1), "batch wait");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->last_ms = ms;
    b->pending = false;
    return batch_status(b);
}

int pf_batch_step(pf_batch* b, int n_steps)
{
    int rc = pf_batch_step_async(b, n_steps);
    if (rc) return rc;
    return pf_batch_wait(b);
}

double pf_batch_last_ms(const pf_batch* b) { return b ? b->last_ms : -1.0; }

int pf_batch_autotune(pf_batch* b, int steps_per_candidate, int* tile_y, int* zchunk, double* ms_per_step)
{
    if (!b || steps_per_candidate < 1) return berr(b, PF_E_ARG, "pf_batch_autotune: bad argument");
    // shape class: precision, median column count bucket, median depth bucket
    std::vector<long long> cols, depth;
    for (const auto& s : b->slots)
        if (s.used) {
            cols.push_back((long long)s.g.nx * s.g.ny);
            depth.push_back(s.g.nz);
        }
    if (cols.empty()) return berr(b, PF_E_STATE, "pf_batch_autotune: empty batch");
    std::nth_element(cols.begin(), cols.begin() + cols.size() / 2, cols.end());
    std::nth_element(depth.begin(), depth.begin() + depth.size() / 2, depth.end());
    const auto key = std::make_tuple(b->prec, (int)std::log2((double)cols[cols.size() / 2] + 1),
                                     (int)std::log2((double)depth[depth.size() / 2] + 1));
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            int rc = pf_batch_set_tile(b, std::get<0>(it->second), std::get<1>(it->second));
            b->pair = std::get<2>(it->second);
            if (tile_y) *tile_y = std::get<0>(it->second);
            if (zchunk) *zchunk = std::get<1>(it->second);
            if (ms_per_step) *ms_per_step = -1.0;
            return rc;
        }
    }
    // every candidate runs real steps (results do not depend on the tile
    // shape), one untimed step first
    double best = 1e300;
    int bty = b->tile_y, bzc = b->zchunk, bpair = 0;
    const bool march = b->march != 0;
    for (int ty : {4, 8, 16})
        for (int zc : {16, 32, 64, 128})
            for (int pr = 0; pr <= ((ty == 8 && (march || !b64(b))) ? 1 : 0); ++pr) {
                if (march && ty != 8) break;   // the march passes run 32 x 8 tiles
                int rc = pf_batch_set_tile(b, ty, zc);
                b->pair = pr;
                if (!rc) rc = pf_batch_step(b, 1);
                if (!rc) rc = pf_batch_step(b, steps_per_candidate);
                if (rc) return rc;
                if (b->last_steps == 0) break;
                const double ms = b->last_ms / (double)b->last_steps;
                if (ms < best) {
                    best = ms;
                    bty = ty;
                    bzc = zc;
                    bpair = pr;
                }
            }
    int rc = pf_batch_set_tile(b, bty, bzc);
    b->pair = bpair;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = std::make_tuple(bty, bzc, bpair);
    }
    if (tile_y) *tile_y = bty;
    if (zchunk) *zchunk = bzc;
    if (ms_per_step) *ms_per_step = best;
    return rc;
}

int pf_batch_track(pf_batch* b, int slot, double out[3])
{
    Slot* sl = get_slot(b, slot);
    if (!sl || !out) return berr(b, PF_E_ARG, "pf_batch_track: bad argument");
    const int nz = sl->g.nz;
    if (nz > b->track_cap) {
        BCK(cudaStreamSynchronize(b->stream), "track sync");
        if (b->d_track) cudaFree(b->d_track);
        b->d_track = nullptr;
        b->track_cap = 0;
        BCK(cudaMalloc(&b->d_track, ((size_t)nz + 1 + 4) * sizeof(unsigned long long)), "track scratch");
        b->track_cap = nz;
    }
    double* res = (double*)(b->d_track + b->track_cap + 1);
    cudaError_t e = b64(b) ? launch_track<double>(sl->bd.d, slot_field(*sl, PF_PHASE_OLD), b->d_track, res, b->stream)
                           : launch_track<float>(sl->bd.d, slot_field(*sl, PF_PHASE_OLD), b->d_track, res, b->stream);
    BCK(e, "pf_batch_track");
    BCK(cudaMemcpyAsync(b->h_out, res, 3 * sizeof(double), cudaMemcpyDeviceToHost, b->stream), "track copy");
    BCK(cudaStreamSynchronize(b->stream), "track sync");
    std::memcpy(out, b->h_out, 3 * sizeof(double));
    return PF_OK;
}

// A checkpoint of one slot, in the format of pf_checkpoint_save (synchronous:
// the caller may remove the slot as soon as this returns).
int pf_batch_checkpoint_save(pf_batch* b, int slot, const char* path)
{
    Slot* sl = get_slot(b, slot);
    if (!sl || !path) return berr(b, PF_E_ARG, "pf_batch_checkpoint_save: bad argument");
    const pf_grid& g = sl->g;
    const size_t row = (size_t)g.nx * b->es;
    const size_t fbytes = row * g.ny * g.nz;
    std::vector<char> host(4 * fbytes);
    for (int i = 0; i < 4; ++i)
        BCK(cudaMemcpy2DAsync(host.data() + i * fbytes, row, slot_field(*sl, kCkptFields[i]),
                              (size_t)sl->bd.d.px * b->es, row, (size_t)g.ny * g.nz, cudaMemcpyDeviceToHost,
                              b->stream),
            "checkpoint copy");
    BCK(cudaStreamSynchronize(b->stream), "checkpoint sync");
    const std::string why = ckpt_write(path, ckpt_header(g, b->prec, sl->st, sl->p), host.data(), fbytes);
    if (!why.empty()) return berr(b, PF_E_STATE, "pf_batch_checkpoint_save: " + why);
    return PF_OK;
}

// Restores a slot (added with the same grid, deck and precision) from a
// checkpoint; the slot continues from the checkpoint's step.
int pf_batch_checkpoint_load(pf_batch* b, int slot, const char* path)
{
    Slot* sl = get_slot(b, slot);
    if (!sl || !path) return berr(b, PF_E_ARG, "pf_batch_checkpoint_load: bad argument");
    std::FILE* f = std::fopen(path, "rb");
    if (!f) return berr(b, PF_E_ARG, std::string("pf_batch_checkpoint_load: cannot open ") + path);
    const pf_grid& g = sl->g;
    CkptHeader h;
    std::string why = ckpt_read_header(f, g, b->prec, sl->p, &h);
    const size_t row = (size_t)g.nx * b->es;
    const size_t fbytes = row * g.ny * g.nz;
    std::vector<char> host;
    if (why.empty()) {
        host.resize(4 * fbytes);
        if (std::fread(host.data(), fbytes, 4, f) != 4) why = "checkpoint shorter than its fields";
    }
    std::fclose(f);
    if (!why.empty()) return berr(b, PF_E_ARG, "pf_batch_checkpoint_load: " + why);
    for (int i = 0; i < 4; ++i)
        BCK(cudaMemcpy2DAsync(slot_field(*sl, kCkptFields[i]), (size_t)sl->bd.d.px * b->es, host.data() + i * fbytes,
                              row, row, (size_t)g.ny * g.nz, cudaMemcpyHostToDevice, b->stream),
            "checkpoint upload");
    BCK(cudaStreamSynchronize(b->stream), "checkpoint sync");
    sl->st = ckpt_state(h);
    return PF_OK;
}

int pf_batch_diagnosticos(pf_batch* b, int slot, double out[5])
{
    Slot* sl = get_slot(b, slot);
    if (!sl || !out) return berr(b, PF_E_ARG, "pf_batch_diagnosticos: bad argument");
    double* res = b->d_part + 592 * kDiagRow;
    cudaError_t e = b64(b) ? launch_diag<double>(sl->bd.d, slot_field(*sl, PF_PHASE_OLD), slot_field(*sl, PF_CONC_OLD),
                                                 slot_field(*sl, PF_TOLD), sl->bd.dpp, b->d_part, 592, res, b->stream)
                           : launch_diag<float>(sl->bd.d, slot_field(*sl, PF_PHASE_OLD), slot_field(*sl, PF_CONC_OLD),
                                                slot_field(*sl, PF_TOLD), sl->bd.dpp, b->d_part, 592, res, b->stream);
    BCK(e, "pf_batch_diagnosticos");
    BCK(cudaMemcpyAsync(b->h_out, res, 6 * sizeof(double), cudaMemcpyDeviceToHost, b->stream), "diag copy");
    BCK(cudaStreamSynchronize(b->stream), "diag sync");
    std::memcpy(out, b->h_out, 5 * sizeof(double));
    const int rc = batch_status(b);
    if (rc != PF_OK) return rc;
    if (b->h_out[5] != 0.0)
        return berr(b, PF_E_NONFINITE, "pf_batch_diagnosticos: " + std::to_string((long long)b->h_out[5]) +
                                           " cells of the slot hold a non-finite phi, c, T or DPP (the run has blown up)");
    return PF_OK;
}

}  // extern "C"
