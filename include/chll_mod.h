/*
 * chll_mod.h -- C ABI of libchll_mod.so, the B200 (sm_100a) chiral
 * Lebwohl-Lasher checkerboard Metropolis library.
 *
 * The first two entry points are the reference's own ctypes boundary and are
 * drop-in replacements for the nvfortran-built libchll_mod.so:
 *   init  <- chll/chll_mod.f90:9-14   (bind(c, name="init")),
 *            bound by ftn_init in chll/chll.py:9-18
 *   run   <- chll/chll_mod.f90:40-48  (bind(c, name="run")),
 *            bound by ftn_run in chll/chll.py:20-36
 * Every scalar is passed by reference, arrays are Fortran-ordered (i fastest)
 * and owned by the caller, exactly as the Fortran interface expects.
 *
 * The chll_* entry points are extensions with the same conventions (plain
 * pointers and sizes, caller-owned buffers).  They return 0 on success and a
 * nonzero CHLL_E* code on failure; chll_last_error() then describes it.  The
 * reference's void entry points report failures the same way (status +
 * message on stderr) instead of aborting the host process.
 *
 * The library runs on the current CUDA device, one stream per lattice, and is
 * not re-entrant across threads for the same lattice; init/run serialise on an
 * internal mutex.
 */
#ifndef CHLL_MOD_H
#define CHLL_MOD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define CHLL_OK 0
#define CHLL_EINVAL 1    /* invalid argument (null pointer, bad size, odd periodic dim) */
#define CHLL_ECUDA 2     /* CUDA runtime error */
#define CHLL_ENOMEM 3    /* device allocation failed */
#define CHLL_EDEVICE 4   /* device-side status word was set */
#define CHLL_ERANGE 5    /* more measurement rows than the caller's buffers hold */

#define CHLL_OPEN 0      /* open boundaries: the reference sweep (chll_mod.f90:371-410) */
#define CHLL_PERIODIC 1  /* periodic boundaries (requires even ni, nj, nk) */

/* Columns of a measurement row (FP64).  0-4 are the reference's m(r,1:5)
 * (chll_mod.f90:99-104): etot, e_excess, paccept, faccept, d. */
#define CHLL_ROW_ETOT 0
#define CHLL_ROW_ETA 1
#define CHLL_ROW_PACCEPT 2
#define CHLL_ROW_FACCEPT 3
#define CHLL_ROW_D 4
#define CHLL_ROW_ENERGY 5        /* total energy, sweep boundary, FP64 */
#define CHLL_ROW_SUM_S 6         /* sum of chiralities */
#define CHLL_ROW_QXX 7           /* raw sums of n_a n_b: xx yy zz xy xz yz (7..12) */
#define CHLL_ROW_ETOT_SUM 13     /* FP64 sum behind column 0 */
#define CHLL_ROW_STEP 14
#define CHLL_ROW_NSITES 15
#define CHLL_ROW_LEN 16

/* ---- reference entry points -------------------------------------------- */

/* Builds the checkerboard index lists: sl1 gets the 1-based F-order indices of
 * sites with (i+j+k) odd (1-based i,j,k), sl2 the rest, each of length nsub.
 * nx..dope are accepted and left untouched, as in the reference.
 * Replaces chll_mod.f90:9-38. */
void init(double* nx, double* ny, double* nz, int* s, int* dope, int* sl1, int* sl2,
          const int* ni, const int* nj, const int* nk, const int* nsub);

/* Runs steps nstart..nstop (one step = director half-sweeps on sl1 then sl2,
 * chirality half-sweeps on sl1 then sl2) on the GPU with open boundaries,
 * adapting d while step < 10000, and measures every nout steps into
 * msteps[r] and m (F-order rows x 5, rows = (1+nstop-nstart)/nout).  Prints
 * the reference's stdout table.  The final state is written back into
 * nx, ny, nz, s; d receives the adapted step size and nsub = N/2.
 * Random numbers: Philox4x32-10 keyed by the seed of chll_set_seed (default 1)
 * and the ordinal of this run() call since that seed was set.
 * sl1, sl2, dope are accepted and not used (the lattice is red/black on the
 * device).  Replaces chll_mod.f90:40-115. */
void run(const int* nstart, const int* nstop, const int* nout, double* nx, double* ny,
         double* nz, int* s, int* dope, int* sl1, int* sl2, double* g, double* KK, double* d,
         double* kbt, const int* ni, const int* nj, const int* nk, int* nsub, int* msteps,
         double* m);

/* ---- errors and seeding ------------------------------------------------- */

/* Status of the last call made on this thread (CHLL_OK if it succeeded). */
int chll_last_status(void);
/* Message of the last failed call on this thread ("" if none). */
const char* chll_last_error(void);
/* Seed of the Philox stream used by run(); resets the run() ordinal. */
void chll_set_seed(uint64_t seed);
/* Library version string. */
const char* chll_version(void);

/* ---- extended run (same semantics as run, explicit options) ------------- */

typedef struct chll_run_config {
  double kT;            /* temperature kbt */
  double K;             /* chiral coupling KK */
  double g;             /* field on the chirality */
  double eps;           /* nematic coupling; 1 reproduces the reference */
  double d;             /* initial proposal amplitude */
  uint64_t seed;        /* Philox key */
  uint32_t replica;     /* Philox counter word 2 */
  int32_t boundary;     /* CHLL_OPEN or CHLL_PERIODIC */
  int64_t adapt_until;  /* d adapted after steps < adapt_until (reference: 10000) */
  int32_t verbose;      /* nonzero: print the reference's stdout table */
  int32_t reserved;
} chll_run_config;

/* run() with explicit options.  m (rows x 5, F-order) and rows16 (rows x
 * CHLL_ROW_LEN, C-order) are optional.  d_out receives the final d.
 * Fails with CHLL_ERANGE (after running) if more steps in nstart..nstop are
 * multiples of nout than the (1+nstop-nstart)/nout rows the buffers hold. */
int chll_run_ex(const chll_run_config* cfg, int nstart, int nstop, int nout, double* nx,
                double* ny, double* nz, int* s, int ni, int nj, int nk, int* msteps, double* m,
                double* rows16, double* d_out);

/* ---- device-resident lattices (bench, autograd, workflows) -------------- */

typedef struct chll_lattice chll_lattice;

typedef struct chll_coupling {
  double kT, K, g, eps;
} chll_coupling;

/* Allocates a red/black float4 lattice of ni x nj x nk sites on the current
 * device (about 16 bytes per site). */
int chll_lattice_create(int ni, int nj, int nk, int boundary, chll_lattice** out);
void chll_lattice_destroy(chll_lattice* lat);
/* Launch stream for all work on this lattice (a cudaStream_t; NULL restores
 * the lattice's own stream; cudaStreamLegacy (0x1) selects the legacy default
 * stream). */
int chll_lattice_set_stream(chll_lattice* lat, void* stream);
/* Sweep form: 0 auto (4 where each of its threads walks at most one unit per
 * pass -- lattices up to about 32^3 -- else 3), 1 the reference's four
 * half-sweeps per step with
 * neighbours read from global memory, 2 the four half-sweeps with row tiles
 * staged in shared memory by bulk copies, 3 the fused two-pass sweep (each
 * pass reads and writes every site once; the colour-0 flips of a step run at
 * the start of the next step's first pass, and after the last step), 4 the
 * fused passes of a whole chunk of steps in one launch of one thread-block
 * cluster whose CTAs meet at the cluster barrier between passes (small
 * lattices, where a pass is mostly launch and grid latency; refused for a slab
 * and with CHLL_ECUDA where no cluster fits).  All give the same chain bit for
 * bit.  chll_lattice_pass runs the staged kernel under 2 and the direct kernel
 * otherwise. */
int chll_lattice_set_kernel(chll_lattice* lat, int kernel);
int chll_lattice_sync(chll_lattice* lat);
/* Random initial state: directors uniform on the sphere, s = +-1 with p=1/2. */
int chll_lattice_init_random(chll_lattice* lat, uint64_t seed, uint32_t replica);
/* F-order FP64 directors and int32 spins, host or device pointers. */
int chll_lattice_upload_f64(chll_lattice* lat, const double* nx, const double* ny,
                            const double* nz, const int* s);
int chll_lattice_download_f64(chll_lattice* lat, double* nx, double* ny, double* nz, int* s);
/* Natural-order (i fastest) float4 (nx, ny, nz, s) records, host or device. */
int chll_lattice_upload_f4(chll_lattice* lat, const float* xyzs);
int chll_lattice_download_f4(chll_lattice* lat, float* xyzs);
/* Red/black storage: colour c array base (device) and its length in float4.
 * For a slab (chll_lattice_create_slab) this is the whole store of nk+3
 * planes, halos included; its own planes start 2*hx*nj float4 in. */
int chll_lattice_storage(chll_lattice* lat, void** colour0, void** colour1, int64_t* per_colour,
                         int32_t* hx);
/* Device control block: d, step, adaptation limit. */
int chll_lattice_set_control(chll_lattice* lat, double d, int64_t step, int64_t adapt_until);
int chll_lattice_get_control(chll_lattice* lat, double* d, int64_t* step, double* paccept,
                             double* faccept);
/* nsweeps full steps from the control block's step, in the form chosen by
 * chll_lattice_set_kernel; every call ends with all trials of its last step
 * done.  Consecutive calls with the same count replay one captured CUDA graph. */
int chll_lattice_sweep(chll_lattice* lat, const chll_coupling* c, uint64_t seed,
                       uint32_t replica, int nsweeps);
/* One pass.  The reference's half-sweeps: 0/1 director trials on colour 0/1,
 * 2/3 chirality flips on colour 0/1 (a step is 0,1,2,3).  The fused passes:
 * 4 colour-0 director trials (first step), 5 the previous step's colour-0
 * flips + colour-0 director trials, 6 colour-1 director trials + colour-1
 * flips (ends the step), 7 the previous step's colour-0 flips (closes the last
 * step): steps t..t+n-1 are 4,6, then 5,6 n-1 times, then 7. */
int chll_lattice_pass(chll_lattice* lat, const chll_coupling* c, uint64_t seed,
                      uint32_t replica, int pass);
/* Device measurement rows: reserve room for n rows, enqueue the FP64
 * observables of the current state into row `slot` without waiting, and read
 * rows [first, first+count) back to the host (waits for the stream). */
int chll_lattice_reserve_rows(chll_lattice* lat, int n);
int chll_lattice_measure(chll_lattice* lat, const chll_coupling* c, int slot);
int chll_lattice_read_rows(chll_lattice* lat, double* rows16, int first, int count);
/* FP64 observables into a host row of CHLL_ROW_LEN doubles. */
int chll_lattice_observe(chll_lattice* lat, const chll_coupling* c, double* row16);
/* Energy adjoint: grad (natural order float4, host or device, may be NULL)
 * receives dE/dn_i (w = 0), tangent-projected if project != 0; out4 (host)
 * receives {E, dE/deps, dE/dK, dE/dh} in FP64. */
/* nsteps of zero-temperature gradient descent, n <- normalise(n - eta *
 * tangent-projected dE/dn), colour 0 then colour 1 each step; chiralities
 * fixed.  Asynchronous on the lattice's stream. */
int chll_lattice_quench(chll_lattice* lat, const chll_coupling* c, double eta, int nsteps);
int chll_lattice_energy_grad(chll_lattice* lat, const chll_coupling* c, float* grad, int project,
                             double* out4);

/* ---- batched replicas (phase-diagram grids) ----------------------------- */

/* One replica of a batch.  Its chain is the one chll_lattice_* would run for
 * the same lattice: Philox key `seed`, counter word 2 `replica`, steps from 1,
 * d adapted while step < 10000.  Replaces the reference's one-process-per-
 * point drivers (scripts/phase_diagram.py:24-31, scripts/g_field0.5.py:24-31). */
typedef struct chll_replica_spec {
  int32_t ni, nj, nk, boundary;
  double kT, K, g, eps, d;
  uint64_t seed;
  uint32_t replica;
  uint32_t reserved;
} chll_replica_spec;

typedef struct chll_batch chll_batch;

/* Columns of a chll_batch_moments row (FP64, 16 per replica). */
#define CHLL_BATCH_NMEAS 0      /* number of measurements */
#define CHLL_BATCH_SUM_E 1      /* sum of e = E/N */
#define CHLL_BATCH_SUM_E2 2
#define CHLL_BATCH_SUM_ETA 3    /* sum of eta = sum(s)/N */
#define CHLL_BATCH_SUM_ETA2 4
#define CHLL_BATCH_SUM_ABS_ETA 5
#define CHLL_BATCH_SUM_S 6      /* sum of S = lambda_max(3/2 <n n> - I/2) */
#define CHLL_BATCH_SUM_S2 7
#define CHLL_BATCH_LAST_E 8
#define CHLL_BATCH_LAST_ETA 9
#define CHLL_BATCH_LAST_S 10
#define CHLL_BATCH_D 11
#define CHLL_BATCH_STEP 12      /* next step number */
#define CHLL_BATCH_PACCEPT 13
#define CHLL_BATCH_FACCEPT 14
#define CHLL_BATCH_STATUS 15
#define CHLL_BATCH_MOM_LEN 16

/* Allocates n replicas of uneven sizes in one device allocation. */
int chll_batch_create(const chll_replica_spec* specs, int n, chll_batch** out);
void chll_batch_destroy(chll_batch* b);
int chll_batch_set_stream(chll_batch* b, void* stream);
int chll_batch_sync(chll_batch* b);
/* Every replica's random initial state from its own (seed, replica). */
int chll_batch_init_random(chll_batch* b);
/* Replica r's state as natural-order float4 records (host or device). */
int chll_batch_upload_f4(chll_batch* b, int r, const float* xyzs);
int chll_batch_download_f4(chll_batch* b, int r, float* xyzs);
/* nsweeps steps of every replica in one persistent cooperative launch
 * (captured once as a CUDA graph, replayed for equal arguments), measuring
 * every measure_every sweeps from sweep measure_from of this call.
 * Asynchronous on the batch's stream. */
int chll_batch_run(chll_batch* b, int nsweeps, int measure_every, int measure_from);
/* Waits, then copies n x CHLL_BATCH_MOM_LEN doubles to the host. */
int chll_batch_moments(chll_batch* b, double* out);
int chll_batch_info(chll_batch* b, int64_t* total_sites, int32_t* nreplicas, int32_t* threads,
                    int32_t* grid);
/* Launch shape: threads per CTA (128, 256, 512) and CTAs per SM (0: all that
 * fit).  Each replica gets CTAs in proportion to its sites. */
int chll_batch_set_tuning(chll_batch* b, int threads, int ctas_per_sm);
/* Replicas run in waves whose float4 state together stays within wave_bytes
 * (0, the default: all replicas in one wave), largest first; each wave gets
 * the whole co-resident grid, in the same launch. */
int chll_batch_set_wave_bytes(chll_batch* b, int64_t wave_bytes);
/* pooled = 1: chll_batch_run sweeps the replicas as pooled passes -- one
 * launch per fused pass over all replicas' units, cut into equal blocks per
 * CTA, the next pass launched as a programmatic dependent (CUDA graphs of
 * measurement-interval chunks) -- instead of the persistent launch with
 * software group barriers; 0 (the default unless chll_batch_autotune chose
 * it): the persistent launch.  The chains are the same either way; the
 * launch shape, waves and pairing apply to the persistent launch only.  No
 * counterpart in the reference, which has no batched launch. */
int chll_batch_set_pooled(chll_batch* b, int pooled);
int chll_batch_get_pooled(chll_batch* b, int* pooled);
/* pair = 1: the replicas of a wave are grouped two by two, by size, and each
 * group's CTAs alternate the two replicas' passes, so a wait at one
 * replica's group barrier overlaps the other replica's pass; 0 (the
 * default): one replica per group.  The chains are the same either way;
 * chll_batch_autotune tries both.  No counterpart in the reference, which
 * has no batched launch. */
int chll_batch_set_pairing(chll_batch* b, int pair);
int chll_batch_get_pairing(chll_batch* b, int* pair);
/* How many polls a replica group's barrier wait makes before it gives up
 * (default 2^24, seconds of waiting; >= 1).  A wait that gives up sets the
 * replica's status word (column 15 of its chll_batch_moments row); every CTA
 * of that replica then leaves the launch at its next barrier, the other
 * replicas run on, and chll_batch_moments returns CHLL_EDEVICE.  The
 * replica's state after such a launch is not usable.  No counterpart in the
 * reference, which has no batched launch. */
int chll_batch_set_wait_limit(chll_batch* b, uint64_t polls);
int chll_batch_get_tuning(chll_batch* b, int32_t* threads, int32_t* ctas_per_sm,
                          int64_t* wave_bytes, int32_t* nwaves);
/* Times every launch shape (threads, CTAs per SM, wave size) for trial_sweeps
 * sweeps from a snapshot of the current state, keeps the fastest and restores
 * the state. */
int chll_batch_autotune(chll_batch* b, int trial_sweeps, int* best_threads, int* best_ctas,
                        double* best_ms);

/* ---- z-slabs: one lattice split over GPUs ---------------------------------- */

/* The slab of global planes z0 .. z0+nkl-1 of an ni x nj x nk lattice (z0 and
 * nkl even, z0 + nkl <= nk), with one halo plane on each side.  Its sites
 * draw the random counters of their global positions, so slabs that exchange
 * halos between passes follow the whole lattice's chain exactly.  A slab is
 * swept pass by pass with chll_lattice_pass codes 4..7 only; each pass only
 * counts accepts: the caller sums the count the pass closes over all slabs
 * (codes 5 and 7: the flip count, 6: the director count; see
 * chll_lattice_counters) and then calls chll_lattice_control_update.  Upload,
 * download, random init and measurement rows act on the slab's own planes
 * (a row's raw sums add up over slabs); the sweep graph, the adjoint, the
 * quench and the analyses take whole lattices only. */
int chll_lattice_create_slab(int ni, int nj, int nk, int z0, int nkl, int boundary,
                             chll_lattice** out);
/* Device address and byte size of one colour's plane of a slab: which = 0 lower
 * halo (global z0-1), 1 first own plane (z0), 2 last own plane (z0+nkl-1),
 * 3 upper halo (z0+nkl).  A plane is hx*nj float4 of one colour. */
int chll_lattice_slab_plane(chll_lattice* lat, int colour, int which, void** ptr,
                            int64_t* bytes);
/* Device address of the control block's pass counters: two uint64 {director
 * accepts, chirality flips}. */
int chll_lattice_counters(chll_lattice* lat, void** ptr);
/* The control update that pass `pass` (4..7) defers on a slab: 5 and 7 close
 * the previous step's flip fraction, 6 the director fraction, d and the step. */
int chll_lattice_control_update(chll_lattice* lat, int pass);
/* Halo exchange inside the passes: every fused pass of colour c also writes
 * the slab's first own plane to lower_c and its last own plane to upper_c
 * (the upper halo of the slab below and the lower halo of the slab above),
 * so no separate exchange is needed between passes, only the ordering that
 * the count sums already give.  NULL = no such neighbour.  32-byte aligned
 * device addresses this GPU can store to: another slab's plane on this GPU
 * (chll_lattice_slab_plane) or a neighbouring GPU's, mapped with
 * chll_ipc_open.  Replaces the caller's halo copies (slab.py TorchHalo).
 * The addresses are used by every later pass: clear them (all NULL) before
 * the memory they point to is freed or unmapped.  Waits for the lattice's
 * stream before changing them. */
int chll_lattice_slab_set_peers(chll_lattice* lat, void* lower0, void* lower1, void* upper0,
                                void* upper1);
/* Copies the first and last own planes of colour `colour` to the peers set
 * above (the halo fill before the first pass). */
int chll_lattice_slab_push(chll_lattice* lat, int colour);
/* IPC export of the lattice's device allocation: the 64-byte
 * cudaIpcMemHandle_t into handle64 and the allocation's address in this
 * process (a plane's offset in it = its address - base).  The exporting
 * process must not destroy the lattice while another process has it mapped. */
int chll_lattice_ipc_handle(chll_lattice* lat, void* handle64, uint64_t* base);
/* Maps an allocation exported by another process (chll_lattice_ipc_handle)
 * into this one: *ptr = its base here.  chll_ipc_close unmaps it. */
int chll_ipc_open(const void* handle64, void** ptr);
int chll_ipc_close(void* ptr);

/* ---- Analysis (the reference's notebook analyses, on the device) ---------- */

/* Shell correlations of calc_n_corr / calc_s_corr (notebooks/paper_plots2.ipynb,
 * cell 0, lines 61-112): over every ordered pair of sites at offset d with
 * |d|^2 < nshells^2 and shell = floor(|d|), gn[shell] is the mean of
 * (n_x . n_{x+d})^2, gs[shell] the mean of s_x s_{x+d} - <s>^2 and counts[shell]
 * the number of pairs.  wrap = 0 keeps both sites inside the lattice (the
 * reference); wrap = 1 takes periodic images.  Arrays of nshells doubles;
 * nshells <= 64.  A shell with no pair gets 0/0 (NaN), as the reference. */
int chll_lattice_shell_corr(chll_lattice* lat, int nshells, int wrap, double* gn, double* gs,
                            double* counts);
/* Chirality projected on an integer direction p = plane[0..2]: hist[m - m_min]
 * is the sum of s over the sites with p . (i+1, j+1, k+1) = m (1-based
 * coordinates, as hero_stripe.py's get_sc).  The structure factor along p,
 * |sum_x s_x exp(-i kv p.(x+1))|^2 / N^2, is |sum_m hist[m] exp(-i kv m)|^2 / N^2.
 * Sets *m_min and *nbins (at most 12288); hist may be NULL to ask the size. */
int chll_lattice_projection(chll_lattice* lat, const int* plane, long long* hist,
                            long long* m_min, int* nbins);

/* ---- energy adjoint without device allocation --------------------------- */

/* Same results as chll_lattice_energy_grad, for callers that cannot let a
 * library call cudaMalloc (a Fortran/OpenACC host whose arrays live in its
 * runtime's device pool, or an application whose own allocator holds nearly
 * all of HBM).  No counterpart in the reference.
 *   colour0, colour1: device red/black lattice arrays, each hx*nj*nk float4
 *     with hx = 2*ceil(ni/4), slot (k*nj + j)*hx + (i>>1) holding site
 *     (i,j,k) of colour (i+j+k)&1, padding slots zero (the layout
 *     chll_lattice_storage exposes);
 *   grad: device, natural order (i fastest) ni*nj*nk float4, may be NULL;
 *   out4: device, 4 doubles {E, dE/deps, dE/dK, dE/dh};
 *   stream: cudaStream_t the work is enqueued on (asynchronous).
 * All intermediates live in one fixed device array of this library (about
 * 4 MiB on every GPU that loads it, held until exit): lattices needing more
 * than 262,144 red/black slots (2*hx*nj*nk; a 64^3 lattice fits) are rejected
 * with CHLL_ERANGE.  colour0, colour1 and grad must be 16-byte aligned and
 * out4 8-byte aligned, all on the current device (or managed), else
 * CHLL_EINVAL before anything is enqueued.  The first call on each device
 * looks up that array's device address; make it before any stream capture
 * (calls outside a capture look it up again, so a device reset leaves no
 * stale address).  Calls share the array: calls whose work overlaps on the
 * GPU race and must be serialised. */
int chll_energy_grad_noalloc(const void* colour0, const void* colour1, int ni, int nj, int nk,
                             int boundary, const chll_coupling* c, int project, float* grad,
                             double* out4, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CHLL_MOD_H */
