/*
 * accel_gpu.h — C-ABI of the B200 tracking engine for Accel+ storage-ring lattices.
 *
 * Every entry point is `extern "C"`, returns an int status (ACCEL_OK == 0, negative on error),
 * takes plain pointers and sizes, and never throws.  Particle state follows the reference's
 * convention: six doubles per particle [x, px, y, py, z, delta]; a lost particle has x = NaN and
 * an aperture code in z (reference accel.cpp:350-354).
 *
 * Pointers flagged "host or device" are classified with cudaPointerGetAttributes: device memory
 * is used in place on the given stream; host memory is staged through the library's device
 * buffers and copied back before the call returns.
 *
 * Reference interfaces replaced (paths inside the reference project, src/lib/accel/):
 *   AccelElement::pass(double*, int)            accel.h:70        -> accel_track (st, ed range)
 *   ALine::pass(double*, int, unsigned, unsigned) accel.h:625      -> accel_track (nturn = 1)
 *   ALine::pass(double*, int), pass(.., nturn)  accel.h:626-627   -> accel_track
 *   ALine::trackDA                              accel.h:628       -> accel_track (loss turns) + host
 *   ALine::trackMA                              accel.h:630       -> accel_track_batched (start offsets)
 *   ALine::getm66                               accel.h:635-637   -> accel_m66
 *   ALine::trackDiffusion / tracktune           accel.h:629,649   -> accel_track_diffusion / _tune
 *   ALine::correcttune / correctchrom           accel.h:644-645   -> accel_correct_tune / _chrom
 *   ALine::deserialize / AccelElement::create   accel.h:68,607    -> accel_lattice_read
 *   ALine::serialize                            accel.h:606       -> accel_lattice_write
 *   AccelElement::setfield / getfield           accel.h:71-72     -> accel_line_set_field / get_field
 *   ALine::set_rad_onoff / set_cavity_onoff /
 *         set_wake_onoff / setenergy            accel.h:613-618   -> accel_line_set_flags / set_energy
 *   ALine::setrfphase()                         accel.h:615       -> accel_line_setrfphase
 *   calc_beam_stat                              utility.h:63      -> accel_beam_stat
 */
#ifndef ACCEL_GPU_H
#define ACCEL_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------ */
#define ACCEL_OK               0
#define ACCEL_E_INVALID       -1  /* bad argument, size or element parameter                   */
#define ACCEL_E_UNSUPPORTED   -2  /* element type or mode the engine does not implement       */
#define ACCEL_E_CUDA          -3  /* a CUDA runtime call failed (message via accel_last_error) */
#define ACCEL_E_NOMEM         -4  /* device or host allocation failed                          */
#define ACCEL_E_IO            -5  /* lattice file could not be opened or parsed                */
#define ACCEL_E_TIMEOUT       -6  /* a bounded device wait ran out (kernel returned early)      */
#define ACCEL_E_NODEVICE      -7  /* no CUDA device visible                                    */
#define ACCEL_E_TOO_LARGE     -8  /* request exceeds a documented fixed capacity               */

/* ---- element types: the names of the reference's type registry (accel.cpp:25-43) ---------- */
#define ACCEL_DRIFT      1
#define ACCEL_QUAD       2
#define ACCEL_CORRECTOR  3
#define ACCEL_APERTURE   4
#define ACCEL_MONITOR    5
#define ACCEL_BEND       6
#define ACCEL_BENDMPOLE  7
#define ACCEL_STRMPOLE   8
#define ACCEL_CAVITY     9
#define ACCEL_WIGTABLE  10   /* kick table by id: accel_wigtable_create */
#define ACCEL_IDEALWIG  11
#define ACCEL_CRABCAV   12
#define ACCEL_RFMULT    13
#define ACCEL_TRANSWAKE 14
#define ACCEL_MATRIX    15
#define ACCEL_SYNCRAD   16
#define ACCEL_LONGWAKE  17   /* no reference counterpart: longitudinal broadband-resonator wake */

#define ACCEL_MAX_MPOLE  10  /* reference MAX_MPOLE, accel.h:48 */

/* radiation flag values (reference accel.h:577-582) */
#define ACCEL_RAD_OFF        0
#define ACCEL_RAD_RAD        1
#define ACCEL_RAD_RADQE      2
#define ACCEL_RAD_LUMP       3
#define ACCEL_RAD_LUMP_DAMP  4
#define ACCEL_RAD_LUMP_QE    5

/*
 * Host-side element descriptor.  One per lattice element, in ring order.  Scalar fields live in
 * f[] with a per-type meaning:
 *   DRIFT      —
 *   QUAD       f0 K
 *   CORRECTOR  f0 KickX, f1 KickY
 *   APERTURE   f0 xmin, f1 xmax, f2 ymin, f3 ymax
 *   MONITOR    f0 Interval, f1 Ratio            (a no-op on the device)
 *   BEND       f0 BendingAngle, f1 e1, f2 e2, f3 K, f4 irho
 *   BENDMPOLE  f0 BendingAngle, f1 e1, f2 e2, f3 energy [MeV], f4 irho; poly_b; max_npole; nslice
 *   STRMPOLE   poly_a, poly_b; max_npole; nslice
 *   CAVITY     f0 Voltage [MV], f1 Frequency [Hz], f2 Phis [rad], f3 Energy [MeV]
 *   TRANSWAKE  f0 Energy, f1 Charge [nC], f2 WakeX, f3 FreqX [GHz], f4 Qx, f5 WakeY, f6 FreqY, f7 Qy
 *   MATRIX     mat[36] row-major
 *   SYNCRAD    f0 Energy, f1 U0, f2 Jx, f3 Jy, f4 EmitX, f5 EmitY, f6 SigDelta, f7 BetaX, f8 BetaY
 *   LONGWAKE   f0 Energy [MeV], f1 Charge [nC], f2 Rs [Ohm], f3 fr [Hz], f4 Q, f5 nbins
 *   CRABCAV    f0 DeVoltX, f1 DeVoltY [MV], f2 Frequency [Hz], f3 Phis, f4 Energy [MeV],
 *              f5 SigPhi, f6 SigdVV (noise from the device's counter-based normals)
 *   RFMULT     f0 Frequency, f1 Phis, f2 Energy, f3 SigPhi, f4 SigdVV; poly_a, poly_b; max_npole
 *   IDEALWIG   f0 lambda, f1 h, f2 type (0 horizontal, 1 vertical), f3 Energy [MeV]; nslice
 *   WIGTABLE   f0 table id (accel_wigtable_create; 0 = none, which tracking rejects); nslice
 * irho is kept as its own field because the reference only refreshes it when BendingAngle is set
 * (accel.h:170, accel.cpp:497,581), not when Length changes.
 * flags: BENDMPOLE / SYNCRAD / IDEALWIG radiation flag (ACCEL_RAD_*), CAVITY / TRANSWAKE /
 * LONGWAKE / CRABCAV on-off.
 */
typedef struct accel_elem_desc {
    int32_t type;
    int32_t nslice;
    int32_t max_npole;
    int32_t flags;
    double  len;
    double  f[12];
    double  poly_a[ACCEL_MAX_MPOLE];
    double  poly_b[ACCEL_MAX_MPOLE];
    double  mat[36];
    char    famname[48];
} accel_elem_desc;

/* field ids for accel_line_set_field / get_field (the reference's setfield names) */
#define ACCEL_F_LENGTH       1
#define ACCEL_F_K            2
#define ACCEL_F_POLYNOMB     3   /* index = order n */
#define ACCEL_F_POLYNOMA     4   /* index = order n */
#define ACCEL_F_NSLICE       5
#define ACCEL_F_MAXNPOLE     6
#define ACCEL_F_ANGLE        7   /* BendingAngle: also refreshes irho, as the reference does */
#define ACCEL_F_E1           8
#define ACCEL_F_E2           9
#define ACCEL_F_VOLTAGE     10
#define ACCEL_F_FREQUENCY   11
#define ACCEL_F_PHIS        12
#define ACCEL_F_ENERGY      13
#define ACCEL_F_KICKX       14
#define ACCEL_F_KICKY       15
#define ACCEL_F_XLIM        16   /* two values */
#define ACCEL_F_YLIM        17   /* two values */

/* track modes */
#define ACCEL_MODE_FUSED  0  /* persistent batched kernel: registers across turns, compaction;
                                the transverse wake (ATransWake, accel.cpp:1603-1657) as z-sorted
                                prefix sums, O(N log N), the same sum in another order */
#define ACCEL_MODE_PLAIN  1  /* one launch per element, state in HBM, reference operation order */
#define ACCEL_MODE_EXACT  2  /* the plain mode's arithmetic, bit-identical to it, with the state
                                in registers over whole turns (one launch per 16 turns, or per
                                range between wake elements); no counterpart in the reference  */

/* state layouts */
#define ACCEL_LAYOUT_AOS  0  /* r[6*i + k]  (the reference's layout) */
#define ACCEL_LAYOUT_SOA  1  /* r[k*N + i]                            */

typedef struct accel_ctx  accel_ctx;   /* one per CUDA device: streams, scratch, tuned tiles */
typedef struct accel_line accel_line;  /* a lattice uploaded to one context                */

/* ---- library / context ------------------------------------------------------------------- */
const char* accel_status_string(int status);
const char* accel_last_error(void);              /* thread-local detail of the last failure   */
int  accel_version(void);
int  accel_device_count(int* n);
/* Handles are released in any order: a context with live lines (or a line with live adjoints)
 * stays usable by those children and is freed when the last of them is destroyed.           */
int  accel_ctx_create(int device, accel_ctx** out);
int  accel_ctx_destroy(accel_ctx* ctx);

/* A bunch spread over several GPUs, one process and one context each (no counterpart in the
 * reference, which runs on one host).  Rank 0 makes an id with accel_nccl_unique_id and sends it
 * to the other ranks (e.g. over torch.distributed); every rank then calls accel_ctx_set_comm with
 * the same id.  From then on each longitudinal wake element of the context's tracking exchanges
 * the bunch's z range, live count and bin counts over NCCL, so every rank kicks its particles
 * with the whole bunch's wake; each transverse wake element (fused mode) all-gathers every rank's
 * (z, x, y) and sums over the whole bunch (the plain and exact modes' pair sum acts within a rank:
 * ACCEL_E_UNSUPPORTED with more than one).  libnccl.so.2 is loaded at run time; without it both calls return
 * ACCEL_E_UNSUPPORTED.  A process holds one libnccl.so.2: where another component (PyTorch) links
 * its own, load that component first and the library uses its copy.  accel_ctx_set_comm blocks
 * until all nranks ranks have called it.  Every rank must then issue the same tracking calls in
 * the same order.                                                                              */
int  accel_nccl_unique_id(unsigned char id[128]);
int  accel_ctx_set_comm(accel_ctx* ctx, const unsigned char id[128], int nranks, int rank);

/* ---- lattice files (host only; no GPU needed) ----------------------------------------------
 * accel_lattice_read follows AccelElement::deserialize (accel.cpp:67-133) and the per-type
 * create() readers; it allocates *elems with malloc (free with accel_lattice_free).          */
int  accel_lattice_read(const char* path, accel_elem_desc** elems, int* n);
int  accel_lattice_parse(const char* text, accel_elem_desc** elems, int* n);
int  accel_lattice_write(const char* path, const accel_elem_desc* elems, int n, int precision);

/*
 * Particle-state checkpoints, lossless (no counterpart in the reference, whose only saved state is
 * the 6-digit text of Do_Track's "Full export", process.cpp:2054-2066, read back by
 * "Distribution: Load f, format=accel-export", process.cpp:1499-1546).  Host arrays, AoS
 * (x px y py z delta per particle).  The file: a 32-byte header ("ACCELST1", uint32 version 1,
 * uint32 flags (bit 0: loss turns present), int64 N, int64 turn), then 6N IEEE-754 doubles, then
 * N int32 loss turns when present; all little-endian.  accel_state_read allocates *r (and
 * *loss_turn, NULL when the file has none) with malloc: release with accel_state_free.
 */
int  accel_state_write(const char* path, const double* r, int64_t N, int64_t turn,
                       const int32_t* loss_turn);
int  accel_state_read(const char* path, double** r, int64_t* N, int64_t* turn, int32_t** loss_turn);
void accel_state_free(void* p);

/*
 * WigTable kick tables (AWigTable, accel.h:403-425; table read/written at accel.cpp:1247-1333).
 * A table is held in a process-wide registry and named from its elements' descriptors by id
 * (f0).  accel_lattice_read / accel_lattice_parse register one table per WigTable entry they read
 * and accel_lattice_write writes it back in the reference's layout.  A line copies the table to
 * its device when it is compiled, so a table may be destroyed once no line will be (re)compiled
 * from descriptors that name it.
 *   mx in 2..101 and my in 2..21 (MAX_WIGTAB_X / MAX_WIGTAB_Y, accel.h:401-402; the
 *   reference's interpolation needs two points per axis, interp_1d.h locate);
 *   xl[mx], yl[my]: the grid, each monotonic (ascending or descending);
 *   xkick, ykick: [my][mx] row-major, kick[i*mx + j] at (xl[j], yl[i]) — the reference's
 *   xkick[i][j] rows.
 * The kicks are interpolated bilinearly (interp2, utility.cpp:174-188), extrapolated from the
 * edge cell outside the grid.  accel_wigtable_get copies out any non-null array.
 */
int  accel_wigtable_create(int mx, int my, const double* xl, const double* yl, const double* xkick,
                           const double* ykick, int32_t* id);
int  accel_wigtable_info(int32_t id, int* mx, int* my);
int  accel_wigtable_get(int32_t id, double* xl, double* yl, double* xkick, double* ykick);
int  accel_wigtable_destroy(int32_t id);
void accel_lattice_free(accel_elem_desc* elems);
int  accel_elem_default(int type, accel_elem_desc* out);   /* the reference's default ctor */

/* ---- lines -------------------------------------------------------------------------------- */
int  accel_line_create(accel_ctx* ctx, const accel_elem_desc* elems, int n, accel_line** out);
int  accel_line_destroy(accel_line* line);
int  accel_line_count(const accel_line* line, int* n);
int  accel_line_get_desc(const accel_line* line, int idx, accel_elem_desc* out);
int  accel_line_set_field(accel_line* line, int idx, int field, int index, const double* value);
int  accel_line_get_field(const accel_line* line, int idx, int field, int index, double* value);
int  accel_line_set_flags(accel_line* line, int rad_flag, int cavity_on, int wake_on);
int  accel_line_set_energy(accel_line* line, double energy_mev);
/* ALine::set_crab_onoff (aline.cpp:441-450): every CrabCav on or off; *count gets their number */
int  accel_line_set_crab_onoff(accel_line* line, int on, int* count);
int  accel_line_setrfphase(accel_line* line, double* phis_out);      /* ALine::setrfphase() */
int  accel_line_set_seed(accel_line* line, uint64_t seed);           /* Philox key for QE     */

/*
 * Track N particles through elements [st, ed) for nturn turns (ALine::pass semantics: a full turn
 * when st == 0 and ed == n).  r: 6N doubles, host or device, in `layout`.  loss_turn (optional,
 * host or device, N int32): -1 for survivors, else the 0-based turn in which x became NaN, which is
 * what the reference's per-turn NaN scan in trackDA records (aline.cpp:646-659).
 * stream: a cudaStream_t; NULL is the legacy default stream.  The work runs on the context's own
 * stream, ordered after the caller's prior work on `stream` and before its later work.
 */
int  accel_track(accel_line* line, double* r, int layout, int N, int st, int ed, int nturn,
                 int32_t* loss_turn, int mode, void* stream);

/*
 * Batched tracking: `ninst` lines (same context) tracked in one persistent launch.  Particles are
 * grouped by instance: instance i owns particles [part_off[i], part_off[i+1]) of the SoA arrays
 * r_soa (6 x Ntot doubles, k-major).  All lines must have the same element count.
 * r_soa and loss_turn (optional, Ntot int32, as in accel_track) are host or device memory each.
 * Device arrays are used in place on `stream` and the call returns without synchronising; a host
 * array is copied in with one cudaMemcpyAsync, tracked in the context's buffer and copied back,
 * and the call returns once the copies are done (page-locked host memory makes those copies
 * asynchronous DMA transfers).
 */
int  accel_track_batched(accel_line* const* lines, int ninst, const int64_t* part_off,
                         double* r_soa, int64_t ntot, int nturn, int32_t* loss_turn,
                         int mode, void* stream);

/* Autotuner control: tile = {block, turns per segment (compaction cadence), variant}, where
 * variant = register-cap variant + 100 x scheduling mode (0: chunks of 32 particles pulled per
 * warp from an atomic counter; 1: a contiguous live-list range per block; 2: blocks of live
 * particles with their instance's element hot lines staged in shared memory).  Register-cap
 * variants 0-5 for modes 0 and 1, 0-2 for mode 2. */
int  accel_autotune(accel_line* const* lines, int ninst, const int64_t* part_off,
                    const double* r_soa, int64_t ntot, int* tile_out3);
int  accel_set_tile(accel_ctx* ctx, int block, int seg_turns, int variant);  /* 0s = auto */
int  accel_get_tile(accel_ctx* ctx, int* tile_out3);
/* The staged schedule (mode 2) waits for each block's shared-memory copy with a bounded number
 * of try_wait probes; a wait that runs out sets an error word, the block waits (bounded again)
 * for its copy in flight and leaves, and the call returns ACCEL_E_TIMEOUT.  probes sets the
 * first wait's limit: 0 the default (2^22), < 0 none (the wait runs out at once, which tests
 * that path).  No counterpart in the reference. */
int  accel_set_stage_wait(accel_ctx* ctx, int probes);

/*
 * One-turn (or [st, ed)) 6x6 transfer matrix around the point (0,0,0,0,0,dpp) (row-major m[36]).
 * method 0: exact tangent map (forward-mode derivative through every element pass);
 * method 1: central differences with step delta, as ALine::getm66 (aline.cpp:900-927).
 */
int  accel_m66(accel_line* line, int st, int ed, double dpp, double delta, int method,
               double* m66);
/* Same, around an arbitrary 6D point r0 (e.g. a closed orbit). */
int  accel_m66_at(accel_line* line, int st, int ed, const double* r0, int method, double delta,
                  double* m66);

/*
 * The exact tangent-map matrix about r0 (as accel_m66_at, method 0) and its exact derivative with
 * respect to one knob: a knob moves the nk coefficients (elem[j], field[j], index[j]) together by
 * the same amount (StrMPole ACCEL_F_POLYNOMB / ACCEL_F_POLYNOMA with index = order, StrMPole
 * ACCEL_F_K = PolynomB[1], Quad ACCEL_F_K), as a magnet family on one power supply does.
 * dm66[6i+j] = d m66[6i+j] / d knob, from hyper-dual numbers through every element pass (second
 * mixed derivatives of the map, no difference in the knob).  It replaces the difference-based
 * knob responses of ALine::calctuneresp / calcchromresp (aline.cpp:1187-1355), which step each
 * family by 1e-5; the tune and chromaticity corrections below are driven by it.
 */
int  accel_m66_knob(accel_line* line, int st, int ed, const double* r0, int nk, const int32_t* elem,
                    const int32_t* field, const int32_t* index, double* m66, double* dm66);

/*
 * Tune and chromaticity correction with two magnet families (ALine::correcttune / correctchrom,
 * accel.h:644-645, aline.cpp:1243-1418): fam1[n1], fam2[n2] are element indices; tune knobs move
 * Quad K or StrMPole PolynomB[1], chromaticity knobs StrMPole PolynomB[2].  *x, *y: the targets
 * in, the achieved values out (tunes from the one-turn matrix about (0,0,0,0,0,dpp) as calctune
 * takes it; chromaticity as the tune change over dpp = +-1e-5, as calcchrom).
 *   method 0: Newton iterations whose 2 x 2 response is the exact knob derivative of the tunes
 *             (accel_m66_knob), until the residual is below 1e-12 (tunes) / 1e-9 (chromaticities)
 *             or stops shrinking, at most maxit; *iterations gets the steps taken;
 *   method 1: the reference's fit: one step of a response built by stepping each family by 1e-5.
 * The families' new coefficients are written into the line.
 */
int  accel_correct_tune(accel_line* line, const int32_t* fam1, int n1, const int32_t* fam2, int n2,
                        double* tunex, double* tuney, int method, int maxit, int* iterations);
int  accel_correct_chrom(accel_line* line, const int32_t* fam1, int n1, const int32_t* fam2, int n2,
                         double* chromx, double* chromy, int method, int maxit, int* iterations);

/*
 * Reverse-mode (adjoint) pair.  Parameters are (element index, field, index) triples
 * (ACCEL_F_POLYNOMB/A of StrMPole, ACCEL_F_K of Quad).
 * accel_adjoint_forward tracks r0 (host or device, AoS, N particles) for nturn turns, keeping a
 * checkpoint of the state every `ckpt_every` turns on the device, and writes r_final.
 * accel_adjoint_backward takes dL/dr_final (AoS, 6N) and returns dL/dr0 (AoS, 6N) and
 * dL/dparams (nparam).  The reverse pass needs every turn's starting state: the forward keeps
 * them all when they fit the tape budget, else each segment is recomputed from its checkpoint.
 * When the Jacobian tape of every turn fits the budget too, the forward writes it as it goes, on
 * a second stream behind the forward's own launches, and returns once it is written; the backward
 * is then one sweep.  Otherwise the backward tapes the Jacobians of a chunk of turns at once, as
 * many as fit the budget, or, when not even one turn fits, reverses turn by turn.  The ways give
 * the same gradient (the last to round-off).  On a line where no element reads z (no cavity),
 * the tapes leave out what only a z component of dL/dr_final would use; a backward call whose
 * dl_drfinal has one writes the tapes again with it first (one more taping pass).
 */
typedef struct accel_adjoint accel_adjoint;  /* holds its line (and context) until destroyed */
int  accel_adjoint_create(accel_line* line, int N, int nturn, int ckpt_every,
                          const int32_t* param_elem, const int32_t* param_field,
                          const int32_t* param_index, int nparam, accel_adjoint** out);
int  accel_adjoint_destroy(accel_adjoint* adj);
int  accel_adjoint_forward(accel_adjoint* adj, const double* r0, double* r_final);
int  accel_adjoint_backward(accel_adjoint* adj, const double* dl_drfinal, double* dl_dr0,
                            double* dl_dparams);
/* Device memory an adjoint created afterwards may give to each of its tapes (the turn starts;
 * the Jacobians, of the whole run or of one chunk of turns); bytes <= 0 restores the default:
 * half of the device memory free when the adjoint is created, at least 4e9.  A smaller budget
 * trades speed for memory.  No counterpart in the reference (which has no reverse mode). */
int  accel_set_adjoint_tape_budget(int64_t bytes);

/* Beam moments of live particles (calc_beam_stat, utility.cpp:387-438): mean[6], sigma[6],
 * cross[6] = <xx'>,<yy'>,<x d>,<x' d>,<y z>,<y' z>; returns the live count in *nlive.  On a
 * context with a communicator (accel_ctx_set_comm) r is this rank's part of a bunch and the
 * moments are the whole bunch's: every rank of the communicator makes the call.              */
int  accel_beam_stat(accel_ctx* ctx, const double* r, int layout, int N, double* mean,
                     double* sigma, double* cross, int* nlive);

/* The same beam moments with no device allocation.  No counterpart in the reference: it exists
 * for callers that cannot let a library allocate: device memory reserved up front by a pool or
 * another framework's caching allocator (a cudaMalloc there fails, or takes memory the pool
 * counted on), and per-turn sampling loops that a cudaMalloc/cudaFree synchronisation would stall.
 *   r    device array of N particles in `layout`, read in place; out  device array of 19 doubles
 *        receiving mean[6], sigma[6], cross[6] and the live count (as a double), in that order.
 *        As in calc_beam_stat, the moments are divided by the live count: with every particle
 *        lost they are NaN and the count is 0.
 *   N    1 .. ACCEL_NOALLOC_STAT_MAX_N; larger N returns ACCEL_E_TOO_LARGE and launches nothing.
 *   stream  where the five small kernels run (NULL = the legacy default stream); the call
 *        returns without synchronising, and `out` is ready when that stream reaches it.
 * Partial sums live in one fixed device array per device (12 * 4096 + 32 doubles), which every
 * call overwrites before reading: nothing in it needs to start at zero.  Because that array is
 * shared, calls on the same device that overlap on the GPU race: issue them on one stream, or
 * order them with events.  The first call on each device does a one-time set-up (the scratch's
 * address via cudaGetSymbolAddress, and the kernels loaded) with that device current; make that
 * first call before beginning any stream capture.  A failed set-up is retried by the next call.
 * A CUDA error already pending from earlier work is reported (ACCEL_E_CUDA) and left pending,
 * and nothing is launched.  It takes no context, so the moments are those of r alone, with no
 * exchange over a communicator.                                                                */
#define ACCEL_NOALLOC_STAT_MAX_N 4194304
int  accel_beam_stat_noalloc(const double* r, int layout, int64_t N, double* out, void* stream);

/* Fundamental frequency (tune) of a real turn-by-turn record, host only: the largest spectral
 * line in [xlow, xhi], refined by golden-section search on the sin^4-windowed projection
 * (the reference's naff, utility.cpp:21-97). */
int  accel_naff(const double* data, int n, double xlow, double xhi, double* nu);

/* Tune diffusion of np starting points (x0[i], y0[i], the other coordinates 0), as
 * ALine::trackDiffusion (accel.h:629, aline.cpp:716-779): each point is tracked for nt - 1 turns,
 * nt the power of two at or above nturn (the points together on the device, in `mode`); NAFF
 * gives the tunes of the first and second halves of the x and y records; nux, nuy receive the
 * first half's, dif = max(-4 ln nt, ln(2 |dnu| / nt)).  A point lost by the end gives NaN in all
 * three and counts -3 in *total (optional), the sum of dif. */
int  accel_track_diffusion(accel_line* line, int nturn, int np, const double* x0, const double* y0,
                           double* nux, double* nuy, double* dif, double xlow, double xhi,
                           double ylow, double yhi, int mode, double* total);
/* Tunes of one starting point (x0, y0) from NAFF over nt turns (nt the power of two at or above
 * nturn), as ALine::tracktune (accel.h:649, aline.cpp:1159-1186). */
int  accel_track_tune(accel_line* line, int nturn, double x0, double y0, double xlow, double xhi,
                      double ylow, double yhi, int mode, double* tunex, double* tuney);

/* Device FP64 FMA throughput micro-benchmark (TFLOP/s, FMA = 2 flops). */
int  accel_fp64_peak(accel_ctx* ctx, double* tflops);
/* The same, and the SM clock (MHz) during the fastest run, from the SM's cycle counter against
 * the global nanosecond timer over one block's loop (sm_mhz may be NULL). */
int  accel_fp64_peak_clocked(accel_ctx* ctx, double* tflops, double* sm_mhz);

/* Device-memory budget of this process's library (no counterpart in the reference, which tracks
 * in host memory).  Every device buffer the library keeps (particle state, element tables,
 * tapes, scratch) is counted; a request that would take the total above the limit fails with
 * ACCEL_E_NOMEM before any cudaMalloc, and the call that needed it returns that status with
 * nothing tracked.  For a GPU shared with other work, and to exercise out-of-memory handling.
 * bytes < 0: no limit (the default).  The limit applies to all devices together and to later
 * requests only; buffers already held stay. */
int  accel_set_device_memory_limit(int64_t bytes);
int  accel_device_memory_held(int64_t* bytes);

/* Number of this library's kernels launched since the context was created. */
int  accel_launch_count(accel_ctx* ctx, int64_t* count);

/* Transverse wake passes of the fused mode that fell back to the pair sum since the context was
 * created.  The z-sorted sum factorises exp(a z_ij); where a * (z_max - z_min) > 600 over the
 * live entries (a bunch many wake lengths long) that would overflow, and each particle then sums
 * over every entry ahead of it: O(N^2) for the N entries of all ranks, 66 ms per pass at 65,536
 * entries and about a minute at 2^20.  No counterpart in the reference, whose pass is always the
 * pair sum (accel.cpp:1603-1657). */
int  accel_transwake_pair_passes(accel_ctx* ctx, int64_t* count);

/* Measurement hook.  When on, every fused-kernel launch inside a tracking graph is bracketed by
 * CUDA events recorded on the stream it runs on; accel_profile_read synchronizes the context's
 * stream and returns, for the most recent tracking call, the summed device time of those
 * launches, their count, and the call's whole device time. */
int  accel_profile_enable(accel_ctx* ctx, int on);
int  accel_profile_read(accel_ctx* ctx, double* fused_ms, int64_t* fused_launches, double* total_ms);

#ifdef __cplusplus
}
#endif
#endif /* ACCEL_GPU_H */
