/*
 * pf3d.h -- C-ABI of the B200 implementation of the coupled explicit time step
 * of the 3-D Al-Cu phase-field model (ileaof/phase-field-project-3D).
 *
 * The reference's hot path is a set of argument-less Fortran subroutines that
 * act on module globals (source/variaveis.f90:3-50), called in a fixed order
 * from the time loop in source/principal.f90:93-259.  This header exports one
 * entry point per subroutine (same name, same meaning), plus a fused step and
 * batched / pooled entry points.  A Fortran caller binds these through
 * ISO_C_BINDING (bind(C), c_loc of its module arrays); a C/C++/Python caller
 * uses them directly.  Plain pointers and sizes only: no CUDA or torch types.
 *
 * Conventions
 *   - Every function returns 0 on success, a negative PF_E* code otherwise;
 *     pf_last_error() gives the message.
 *   - Fields are Nx*Ny*Nz arrays in Fortran order (i fastest), 1-based (i,j,k)
 *     in every index argument, exactly like the reference arrays.
 *   - A context owns its device buffers; the caller owns host arrays.
 *   - Each context is driven by one host thread (the reference calls its
 *     subroutines from serial code only) and runs on one CUDA stream.
 *   - Work is stream-ordered; pf_download, pf_diagnosticos, pf_probe and
 *     pf_sync block until the result is on the host.
 */
#ifndef PF3D_H
#define PF3D_H

#ifdef __cplusplus
extern "C" {
#endif

#define PF3D_VERSION 1

/* status codes */
#define PF_OK 0
#define PF_E_ARG (-1)      /* invalid argument / unsupported size          */
#define PF_E_CUDA (-2)     /* CUDA runtime error (message in pf_last_error) */
#define PF_E_NOMEM (-3)    /* device allocation refused or over budget      */
#define PF_E_STATE (-4)    /* call not valid in the current state           */
#define PF_E_NODEV (-5)    /* no CUDA device visible                        */
#define PF_E_NONFINITE (-7) /* the diagnostics found cells whose phi, c, T
                              or DPP is not finite (the run has blown up);
                              the five values are still returned          */
#define PF_E_KERNEL (-6)   /* a kernel reported a failure in the context's
                              status word (a TMA plane load that did not
                              arrive within its bounded wait); reported by
                              the next pf_sync / pf_download / diagnostics  */

/* field ids: the seven resident arrays of source/principal.f90:61-63 */
#define PF_PHASE_OLD 0     /* phase_field_old */
#define PF_PHASE_NEW 1     /* phase_field_new */
#define PF_CONC_OLD 2      /* conc_soluto_old */
#define PF_CONC_NEW 3      /* conc_soluto_new */
#define PF_TOLD 4          /* TOLD            */
#define PF_TNEW 5          /* TNEW            */
#define PF_DPP 6           /* DPP             */

/* storage / arithmetic precision of a context */
#define PF_FP64 64         /* plain form: FP64 end to end, reference arithmetic  */
#define PF_FP32 32         /* FP32 fields and stencils, FP64 scalars and sums    */

/* boundary treatment */
#define PF_BC_REFERENCE 0  /* plane-copy decoration of the reference (default)   */

/* Grid: Nx, Ny, Nz (>= 5 each) and the spacings dx, dy, dz [m]. */
typedef struct pf_grid {
    int nx, ny, nz;
    double dx, dy, dz;
} pf_grid;

/*
 * Physical and numerical parameters: the entrada.dat deck, by the reference's
 * names (source/entrada.f90:19-89).  Ke, Sigma, Beta and ajuste are REAL(4)
 * in the reference (source/variaveis.f90:28) and stay float here, because
 * their single-precision rounding enters W0/E0 and M0.
 */
typedef struct pf_params {
    double Tm;             /* melting temperature [K]                             */
    double T0;             /* initial temperature [K]                             */
    double delta_H;        /* latent heat [J/m^3]                                 */
    double M0;             /* interface mobility used by step 1 (then auxiliar)   */
    double Cp_s;           /* heat capacity used by temperatura (cp = cp_s)       */
    double D;              /* heat-equation diffusivity; the reference never
                              assigns its module variable D, so the deck value 0
                              reproduces it                                       */
    double AAA;            /* noise amplitude as read from the deck (before the
                              dt rescale of entrada.f90:179-185)                  */
    double DELTA_EPSLON;   /* anisotropy strength                                 */
    double D_sol, D_liq;   /* solute diffusivities [m^2/s]                        */
    float  Ke;             /* partition coefficient (REAL(4))                     */
    double Me;             /* liquidus slope [K/mol fraction]                     */
    double Vm;             /* molar volume [m^3/mol]                              */
    double R;              /* gas constant                                        */
    double C0;             /* initial solute concentration                        */
    double Thin_Interface; /* Lambda = Thin_Interface * dx                        */
    float  Sigma;          /* surface energy (REAL(4))                            */
    float  Beta;           /* kinetic coefficient (REAL(4))                       */
    float  ajuste;         /* mobility adjustment (REAL(4))                       */
    double TP;             /* isothermal TP line; replaced by T0 if taxa_resfr>0   */
    double taxa_resfr;     /* cooling rate [K/s]; TP = T0 - taxa*dt*it            */
    int    n_varreduras;   /* phase sweeps per step (>= 1)                        */
    int    h_quintico;     /* 1 = quintic h(phi), 0 = cubic                       */
    int    ruido_tipo;     /* 0 cell noise >= 0, 1 zero-mean cell, 2 smooth       */
    int    bc;             /* PF_BC_REFERENCE                                     */
    double stoptime;       /* [s]; 0 = no stop test (driver only)                 */
    int    WriteFileD_timeCounter; /* output cadence (driver only)               */
} pf_params;

/* Quantities derived once at set-up (entrada.f90:159-185, W0_E0.f90). */
typedef struct pf_derived {
    double DELTA_T;        /* dt = dx^2 / (7.5 D_liq)                             */
    double AAA;            /* effective noise amplitude after the dt rescale      */
    double Lambda;         /* Thin_Interface * dx                                 */
    double W0, E0;         /* from the W0_E0 fixed-point scan                     */
    long   w0e0_iterations;
} pf_derived;

/* Host-side step state that the reference keeps in module scalars. */
typedef struct pf_state {
    int    it;             /* last completed step (0 before the first)            */
    double TP;             /* current TP                                          */
    double M0;             /* mobility the next phase sweep will use              */
    double Cs_eq, Cl_eq;   /* from the last phase sweep                           */
    float  time;           /* REAL(4) simulated time (principal.f90:96)           */
} pf_state;

typedef struct pf_ctx pf_ctx;

/* ---- library / context lifecycle ------------------------------------- */
int         pf_version(void);
const char* pf_last_error(const pf_ctx* ctx);   /* ctx may be NULL           */
/* Bytes of device memory a context of this grid and precision holds.       */
long long   pf_ctx_bytes(const pf_grid* g, int precision);
int pf_create(const pf_grid* g, const pf_params* p, int precision, pf_ctx** out);
int pf_destroy(pf_ctx* ctx);
int pf_get_derived(const pf_ctx* ctx, pf_derived* out);
int pf_get_state(const pf_ctx* ctx, pf_state* out);
int pf_set_state(pf_ctx* ctx, const pf_state* st);
int pf_sync(pf_ctx* ctx);
/* Run the context's work on the caller's CUDA stream (a cudaStream_t passed
   as void*; NULL returns to the context's own stream).                     */
int pf_set_stream(pf_ctx* ctx, void* stream);

/* options (pf_set_option / pf_get_option) */
#define PF_OPT_FUSED 1     /* 1 (default): pf_step uses the fused kernels;
                              0: it calls the per-subroutine kernels        */
#define PF_OPT_TILE_Y 2    /* fused tile height: 4, 8 (default) or 16       */
#define PF_OPT_ZCHUNK 3    /* z planes per fused CTA (0 = whole column)     */
#define PF_OPT_KTIMING 4   /* 1: time every fused launch with CUDA events   */
#define PF_OPT_PAIRED 5    /* two cells per thread on 32 x 8 fused tiles
                              (same results): 1 (default) in FP32, where it
                              is faster; 2 in both precisions; 0 never      */
#define PF_OPT_KERNEL 6    /* fused passes on 32 x 8 tiles: 1 (default) TMA
                              plane loads on mbarriers, uniform per-cell
                              arithmetic with fan-out boundary stores; 0 the
                              element-wise cp.async passes.  Same results.  */
#define PF_OPT_NSLOT 7     /* window mode of the TMA passes: 3 (3-plane
                              node windows), 4 (4-plane windows) or 5 (the
                              own column's values carried in registers along
                              z, 3-plane windows); one barrier a plane in
                              each; 0 (default) = 3.  Same results.         */
int pf_set_option(pf_ctx* ctx, int opt, int value);
int pf_get_option(const pf_ctx* ctx, int opt, int* value);
/* With PF_OPT_KTIMING on: launches and summed device milliseconds of the
   first (heat + sweep 1) and last (sweep 2 + solute) fused kernels since
   the last reset.  Synchronises the context's stream.                      */
int pf_kernel_times(pf_ctx* ctx, long* n_first, double* ms_first, long* n_last, double* ms_last, int reset);

/* ---- data residency (principal.f90:60-64, :182, :248, :268-272) ---------- */
/* host array: Nx*Ny*Nz doubles, Fortran order.  FP32 contexts convert.     */
int pf_upload(pf_ctx* ctx, int field, const double* host);
int pf_download(pf_ctx* ctx, int field, double* host);
/* read one cell, 1-based (the progress print of equacao_campo_fase.f90:174) */
int pf_probe(pf_ctx* ctx, int field, int i, int j, int k, double* value);

/* ---- host scalar set-up, FP64 (no device needed) ---------------------- */
/* W0_E0.f90:10-31: fixed-point scan for W0 and E0.                        */
int pf_w0_e0(const pf_grid* g, const pf_params* p, double* W0, double* E0, long* iterations);
/* auxiliar.f90:12-42: M0 from TP and the equilibrium compositions.        */
int pf_auxiliar_scalar(const pf_params* p, double E0, double W0, double TP,
                       double Cs_eq, double Cl_eq, double* M0);

/* ---- one entry point per reference subroutine ------------------------- */
/* temperatura.f90: TNEW = TOLD, then temp_body.inc on 2..N-1, with the
   given TP (the reference passes the TP of the previous step).            */
int pf_temperatura(pf_ctx* ctx, double TP);
/* equacao_campo_fase.f90: Cs_eq/Cl_eq from TP, phase_field_new = old,
   phase_body.inc on 3..N-2 (noise index it), boundary decoration.  Cs_eq
   and Cl_eq may be NULL.                                                  */
int pf_equacao_campo_fase(pf_ctx* ctx, int it, double TP, double M0,
                          double* Cs_eq, double* Cl_eq);
/* principal.f90:128-150: phase_field_old = phase_field_new (between sweeps) */
int pf_copy_phase_new_to_old(pf_ctx* ctx);
/* concentracao_soluto.f90: conc_body.inc on 2..N-1, conc_soluto_old = new,
   boundary decoration of conc_soluto_new from conc_soluto_old.            */
int pf_concentracao_soluto(pf_ctx* ctx);
/* auxiliar.f90 with the context's E0/W0/parameters.                       */
int pf_auxiliar(const pf_ctx* ctx, double TP, double Cs_eq, double Cl_eq, double* M0);
/* diagnosticos.f90: out = {L2_phi, phi_max, phi_min, solute_total,
   free_energy} of phase_field_new / conc_soluto_new.  Watchdog: the same
   reduction counts the cells where phi, c, TNEW or DPP is not finite (the
   clamp of the phase update turns a NaN update into 1, so a blow-up can
   show only in DPP and T); if any, the call returns PF_E_NONFINITE with out
   still filled (max/min NaN when phi holds the NaN).                       */
int pf_diagnosticos(pf_ctx* ctx, double out[5]);
/* principal.f90:200-226: old <- new for phi, T and c.  Done by exchanging
   buffers: afterwards the "new" arrays hold the previous "old" data until
   the next subroutine overwrites them (the reference's loop reads none of
   them in between).                                                        */
int pf_swap(pf_ctx* ctx);

/* No counterpart in the reference.  pf_diagnosticos without any device
   allocation, for callers that cannot let a library allocate device memory
   (a program whose device memory belongs to another runtime, such as an
   OpenMP target-offload build that passes `use_device_addr` pointers of its
   mapped fields, or a solver under a fixed device-memory budget).  The
   caller passes its own device fields (Fortran order, row pitch `pitch` >=
   nx elements, PF_FP64 doubles or PF_FP32 floats) and receives the five
   values of pf_diagnosticos in out[5] (host); the call waits on `stream`
   for them before it returns.  Scratch is a static device array of
   PF_NOALLOC_MAX_PLANES rows of partials (about 256 KiB per device, held
   until the process exits); each plane is reduced in one or more rows, so
   nz above that limit is rejected with PF_E_ARG.  The first call on each
   device looks up the array's device address, so make it before any stream
   capture.  All calls share the array: calls whose work overlaps on the GPU
   race.  `stream` is a cudaStream_t or NULL.                               */
#define PF_NOALLOC_MAX_PLANES 4096
int pf_diagnosticos_noalloc(const void* phase_field, const void* conc_soluto, int nx, int ny, int nz,
                            int pitch, int precision, double dx, double dy, double dz, double E0,
                            double W0, void* stream, double out[5]);

/* Seeded synthetic initial state written on the device into the old fields
   and DPP (the reference fills its fields on the host, entrada.f90:226-262):
   a solid slab k <= 4 carrying hemispherical bumps of radius 3 cells at the
   1-based (i, j) centres sites[2*b], sites[2*b+1]; phi = (1-tanh(2d/w))/2
   with d the signed distance to slab U bumps and w = Thin_Interface cells;
   c = C0 (1 - (1 - Ke) phi); T = T0; DPP = 0.  At most 4096 bumps.        */
int pf_init_seeded(pf_ctx* ctx, int n_bumps, const double* sites);

/* ---- tracking, checkpoints, moving frame ------------------------------ */
/* Solidification tracking on the device, no field copied to the host:
   out = {solid fraction mean(phi >= 0.5), tip position, solid cells} of
   phase_field_old (the state after the last step).  Tip position = the
   highest 1-based plane k where some (i, j) column has phi >= 0.5, plus the
   linear interpolation to the 0.5 crossing between the maxima of planes k
   and k+1 (k itself when k = nz; 0 with no solid): the tip height of the
   reference's run log (docs/run6/README.md:54-62) as karma/karma3d.f90:
   291-298 tracks it.  Equal bit for bit to the same metric on the
   downloaded field.                                                        */
int pf_track(pf_ctx* ctx, double out[3]);

/* Binary checkpoint of the domain's state (phase_field_old, conc_soluto_old,
   TOLD, DPP in the context's precision, plus pf_state): no counterpart in
   the reference, whose only restart is its 8-digit Tecplot text
   (saida.f90:20-54 read back by entrada.f90:284-321).  A run continued from
   a checkpoint gives the same bits as the run never stopped.
   pf_checkpoint_save is asynchronous: it enqueues the device-to-host copy on
   the context's stream and returns; a host thread writes the file once the
   copy has landed, while the caller keeps stepping.  pf_checkpoint_wait
   waits for that writer and returns its status; a second save, a load and
   pf_destroy wait for it too.  pf_checkpoint_load is synchronous; the
   file's grid and precision must be the context's.                        */
int pf_checkpoint_save(pf_ctx* ctx, const char* path);
int pf_checkpoint_wait(pf_ctx* ctx);
int pf_checkpoint_load(pf_ctx* ctx, const char* path);

/* Moving frame on the device, replacing the reference's manual restart with
   a shift (entrada.f90:284-321, tipo_inicial = 4 with k_desl = R_semente):
   phase_field_old and conc_soluto_old move down by k_desl planes (plane k
   takes plane k + k_desl); the k_desl top planes become liquid, phi = 0 with
   each column's c of the former top plane; conc_soluto_new = conc_soluto_old,
   phase_field_new = 0, TOLD = TNEW = T0 and DPP = 0 (entrada's initial fill,
   entrada.f90:239-262).  The pf_state is left alone (the reference's restart
   starts a new run: set it with pf_set_state).  0 <= k_desl < nz, else
   PF_E_ARG (entrada.f90:292).                                             */
int pf_shift_frame(pf_ctx* ctx, int k_desl);

/* ---- fused step ------------------------------------------------------- */
/* Runs n_steps whole iterations of principal.f90:93-226 (temperatura, TP
   ramp, n_varreduras sweeps, solute, auxiliar, swap) with the fused
   kernels, starting from the context's pf_state.  Results equal the
   sequence of per-subroutine calls above.                                 */
int pf_step(pf_ctx* ctx, int n_steps);
/* Same, and also fills out[5] with the diagnostics of the final state
   (PF_E_NONFINITE, out filled, if that state holds a non-finite value).   */
int pf_step_diag(pf_ctx* ctx, int n_steps, double out[5]);

/* ---- batches of independent domains ---------------------------------- */
/* Many domains of one precision, each with its own grid, deck and step
   count, advanced together: one persistent launch per pass over a work list
   of (domain, tile) items, K steps per captured CUDA graph.  Domains join
   (pf_batch_add) and leave (pf_batch_remove) between pf_batch_step calls
   under a device-memory budget; each keeps the reference's per-domain step
   semantics of pf_step, and its results are the same bits as pf_step's on
   the same domain.  All domains of a batch use the same n_varreduras (1/2). */
typedef struct pf_batch pf_batch;
int pf_batch_create(int precision, long long budget_bytes, int max_domains, pf_batch** out);
int pf_batch_destroy(pf_batch* b);
int pf_batch_set_stream(pf_batch* b, void* stream);
long long pf_batch_bytes_used(const pf_batch* b);
int pf_batch_count(const pf_batch* b);
/* PF_E_NOMEM when the domain does not fit the budget or no slot is free    */
int pf_batch_add(pf_batch* b, const pf_grid* g, const pf_params* p, int* slot);
int pf_batch_remove(pf_batch* b, int slot);
int pf_batch_upload(pf_batch* b, int slot, int field, const double* host);
int pf_batch_download(pf_batch* b, int slot, int field, double* host);
int pf_batch_init_seeded(pf_batch* b, int slot, int n_bumps, const double* sites);
/* the slot stops advancing once it has completed target_it steps (0: never) */
int pf_batch_set_target(pf_batch* b, int slot, long long target_it);
int pf_batch_get_state(const pf_batch* b, int slot, pf_state* out);
/* the step count (pf_state.it) of slots 0 .. n-1 in one call, -1 for a
   free slot: what a serving loop polls every quantum                      */
int pf_batch_progress(const pf_batch* b, int* it, int n);
/* advance every active slot by up to n_steps steps                        */
int pf_batch_step(pf_batch* b, int n_steps);
/* the same without waiting: the steps are queued on the batch's stream (the
   host state of every slot is already advanced); pf_batch_wait waits for
   them.  Two batches on their own streams so run at the same time.        */
int pf_batch_step_async(pf_batch* b, int n_steps);
int pf_batch_wait(pf_batch* b);
/* device milliseconds of the last pf_batch_step call (all its graphs)      */
double pf_batch_last_ms(const pf_batch* b);
int pf_batch_set_tile(pf_batch* b, int tile_y, int zchunk);
/* 32 x 8 tiles: 1 runs two cells per thread (same results), 0 one.  The
   TMA passes pair cells in either precision, except in batches with the
   smooth noise; the cp.async passes pair FP32 batches without the smooth
   noise or heat diffusion only                                             */
int pf_batch_set_paired(pf_batch* b, int paired);
/* Which fused passes a batch runs (same results): kernel 1 (default) the
   TMA-staged passes on 32 x 8 tiles, 0 the element-wise cp.async passes;
   nslot as PF_OPT_NSLOT (0 = 3)                                           */
int pf_batch_set_kernel(pf_batch* b, int kernel, int nslot);
/* Autotuner: times every tile shape x z-chunk (16, 32, 64, 128) x one or
   two cells per thread -- tile heights 4, 8 and 16 for the cp.async passes,
   32 x 8 for the TMA passes -- on real steps (the results do not depend on
   these choices; each candidate advances the batch by 1 +
   steps_per_candidate steps), keeps the fastest and caches it per shape
   class (precision, median column size and depth)                         */
int pf_batch_autotune(pf_batch* b, int steps_per_candidate, int* tile_y, int* zchunk, double* ms_per_step);
/* pf_diagnosticos of one slot's state (the watchdog as there)             */
int pf_batch_diagnosticos(pf_batch* b, int slot, double out[5]);
/* pf_track of one slot                                                    */
int pf_batch_track(pf_batch* b, int slot, double out[3]);
/* Checkpoint of one slot in pf_checkpoint_save's format (synchronous, so a
   server may remove the slot right after it, e.g. to preempt the request);
   load restores a slot added with the same grid, deck and precision.      */
int pf_batch_checkpoint_save(pf_batch* b, int slot, const char* path);
int pf_batch_checkpoint_load(pf_batch* b, int slot, const char* path);

/* ---- the quantitative Karma model (karma/karma3d.f90) ----------------- */
/* The reference's second model: isothermal free growth of a dilute binary
   alloy (Karma PRL 87 115701 2001; Echebarria, Folch, Karma & Plapp PRE 70
   061604 2004) with phi in [-1, 1], the dimensionless supersaturation U,
   cubic anisotropy eps4, the anti-trapping current and mirror (zero-flux)
   faces, in units of the interface width W and time tau0.  The namelist of
   karma.nml by its names (karma3d.f90:80-95); the reference's domain is
   N^3 (nx = ny = nz = N), any extents are accepted here.                  */
typedef struct pf_karma_params {
    int    nx, ny, nz;
    double lambda;         /* coupling constant, W/d0 = lambda/a1              */
    double eps4;           /* cubic anisotropy of the interface energy         */
    double dx;             /* cell size [W]                                    */
    double dt;             /* time step [tau0]                                 */
    double R0;             /* seed radius [W]                                  */
    double Fnoise;         /* noise amplitude of the phase equation            */
    double k, Tm, mliq, C0, TP, sigma, dH, Dl;   /* alloy (entrada.dat data)   */
} pf_karma_params;

/* dimensional scales of karma3d.f90:118-124                                */
typedef struct pf_karma_derived {
    double D;              /* a2 lambda (dimensionless diffusivity)           */
    double cl0, Omega;     /* liquidus concentration at TP; supersaturation   */
    double Gam, d0;        /* Gibbs-Thomson coefficient; capillary length [m] */
    double W, tau0;        /* interface width [m]; relaxation time [s]        */
} pf_karma_derived;

#define PF_KARMA_PHI  0
#define PF_KARMA_U    1
#define PF_KARMA_DPHI 2    /* dphi/dt of the last step (download only)       */

typedef struct pf_karma pf_karma;
int pf_karma_derived_of(const pf_karma_params* p, pf_karma_derived* out);
int pf_karma_create(const pf_karma_params* p, int precision, pf_karma** out);
int pf_karma_destroy(pf_karma* k);
int pf_karma_set_stream(pf_karma* k, void* stream);
/* steps done (the noise of step n uses it = n, karma3d.f90:161)            */
int pf_karma_get_it(const pf_karma* k, int* it);
int pf_karma_set_it(pf_karma* k, int it);
/* interior cells, Fortran order (nx*ny*nz doubles)                         */
int pf_karma_upload(pf_karma* k, int field, const double* host);
int pf_karma_download(pf_karma* k, int field, double* host);
/* karma3d.f90:130-144 on the device: an eighth of a sphere of radius R0 at
   the corner (phi = -tanh((r - R0)/sqrt 2)), U = -Omega; it = 0            */
int pf_karma_seed(pf_karma* k);
/* n_steps iterations of karma3d.f90:160-287 (mirror faces, phase equation,
   U equation with the anti-trapping current, clamp and advance); in FP64
   every operation is the reference's, in its order                       */
int pf_karma_step(pf_karma* k, int n_steps);
/* karma3d.f90:290-296: the largest i with phi(i,1,1) > 0 and with
   phi(i,i,i) > 0 (1-based; 0 if none), evaluated on the device             */
int pf_karma_tip(pf_karma* k, int* tip_x, int* tip_d);
int pf_karma_sync(pf_karma* k);

/* ---- self-check of the fast form's own FP64 logarithm ------------------
   The fused FP64 kernels take log(CL/(1-CL)) and log|...| of
   phase_body.inc / soluto_body.inc with this library's logarithm (atanh
   series with argument reduction) instead of the CUDA library's.  This
   evaluates both on the device for n host values: own[i] = the fused
   kernels' log(x[i]), lib[i] = CUDA's log(x[i]).  No reference routine.   */
int pf_math_log(const double* x, long long n, double* own, double* lib);

#ifdef __cplusplus
}
#endif
#endif /* PF3D_H */
