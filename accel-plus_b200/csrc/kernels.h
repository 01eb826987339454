// kernels.h — launch interface of the CUDA translation units (host-callable).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "engine.h"

namespace accel {

// Particle state is SoA: coordinate k of particle p at st[k * ntot + p].
struct TrackParams {
    const DevElem* tables;   // concatenated element tables
    const int32_t* tbl_off;  // [ninst] record offset of each instance's table (nullptr: 0)
    const int32_t* pinst;    // [ntot] instance of each particle (nullptr: all 0)
    double* st;              // SoA state
    int64_t ntot;
    int32_t* loss_turn;      // [ntot]; -1 alive
    const int32_t* live;     // live list (fused) — entries index st
    const int32_t* nlive;    // device count of live entries
    int32_t* chunk_ctr;      // fused: atomic chunk counter, zero at launch
    int32_t* err;            // error word (bounded waits)
    int32_t* lost_flag;      // set to 1 by a launch that loses a particle (may be null)
    int e0, e1;              // element range
    int nturn;               // turns in this launch (fused)
    int turn0;               // turn index (loss record) of the launch's first turn
    const int32_t* turn_dev; // device turn counter added to turn0 and rng_turn0 (may be null)
    int rng_turn0;           // turn offset fed to the QE counter
    int sched;               // fused: 0 chunks pulled per warp from an atomic counter,
                             //        1 contiguous live-list range per block (L1 keeps fewer tables)
    const int32_t* rng_base; // device: QE turn base of the line (advanced per call)
    uint64_t seed;
    int32_t* tw_pair_passes; // transverse wake passes that fell back to the pair sum (may be null)
    int stage_wait;          // staged schedule: try_wait probes of a stage's first wait (0: the
                             // default limit; < 0: none, the wait counts as run out at once)
};

// ---- fused (kern_fused.cu) ----------------------------------------------------------------
constexpr int kNumFusedVariants = 6;
// 0: chunks pulled per warp from an atomic counter; 1: a contiguous live-list range per block;
// 2: per-block tasks with the instance's element hot lines staged in shared memory (staged
//    variants, their own (block, min blocks) table)
constexpr int kNumSched = 3;
constexpr int kSchedStaged = 2;
constexpr int kNumStagedVariants = 3;
struct VariantInfo { int block; int min_blocks; };
VariantInfo fused_variant_info(int v);
int fused_blocks_per_sm(int variant);                     // occupancy at the variant's block
void launch_fused(const TrackParams& p, int variant, int grid, cudaStream_t s);
VariantInfo staged_variant_info(int v);
int staged_blocks_per_sm(int v, int ne);  // resident blocks with ne hot lines each (0: does not fit)
void launch_fused_staged(const TrackParams& p, int v, const void* hot, int ne, int grid, cudaStream_t s);
// the first 128-byte line of each of nrec records, contiguous (the staged variant's source)
void launch_extract_hot(const DevElem* tbl, int64_t nrec, void* hot, cudaStream_t s);
// Stable compaction, in place (live == the list it compacts).  Resets the chunk counter and adds
// `turns` to the device turn counter.  With lost_flag, the list is scanned only when the flag is
// set (a particle was lost since the last compaction), and the flag is cleared.
void launch_compact(int32_t* live, int32_t* nlive, const double* x, int32_t* chunk_ctr, int32_t* turn_ctr,
                    int turns, int32_t* lost_flag, cudaStream_t s);
void launch_init_live(const double* x, int64_t n, int32_t* loss_turn, int32_t* live, int32_t* nlive,
                      int32_t* chunk_ctr, int init_loss, cudaStream_t s);
void launch_aos_to_soa(const double* aos, double* soa, int64_t n, cudaStream_t s);
void launch_soa_to_aos(const double* soa, double* aos, int64_t n, cudaStream_t s);
void launch_fill_i32(int32_t* p, int32_t v, int64_t n, cudaStream_t s);
void launch_copy_i32(const int32_t* src, int32_t* dst, int64_t n, cudaStream_t s);
// collective elements on the live list (one instance only)
void launch_longwake(const TrackParams& p, const DevElem* e_dev, const DevElem& e_host,
                     double* scratch, int32_t* iscratch, cudaStream_t s);
void launch_transwake(const TrackParams& p, const DevElem* e_dev, const DevElem& e_host,
                      double* xsnap, cudaStream_t s);
size_t longwake_scratch_doubles(int nbins);
// transverse wake in O(N log N) (kern_tw.cu): z-sorted prefix sums of the factorised resonator
// wake.  Each rank offers `slots` entries (z, x, y; z = -inf for none), at least its particle
// count and the same on every rank; the sum runs over all ranks' entries (`nranks` x `slots`),
// gathered between the two stages, with the charge per particle Ne / ntot_all.  Scratch from
// tw_sorted_scratch_bytes, allocated before any capture.
struct TwLayout {
    int64_t slots, total;             // entries per rank, over all ranks
    double *key_s, *x_s, *y_s;        // this rank's entries (gather send buffers)
    double *key_g, *x_g, *y_g;        // all ranks' entries (gather receive buffers)
    double* key_sorted;
    int32_t *val_in, *val_sorted;     // entry index, rank * slots + slot
    void *terms, *prefix;             // four weighted sums per sorted entry, their in-tile scan
    void* tile_off;                   // and the tiles' offsets
    int32_t* nvalid;                  // [0] this rank's live entries, [1] all ranks'
    void* tmp;
    size_t tmp_bytes;
};
// gather: the entries are exchanged between the stages (a communicator is set); without it the
// rank's entries are the whole list
size_t tw_sorted_scratch_bytes(int64_t slots, int nranks, bool gather);
TwLayout tw_layout(void* scratch, int64_t slots, int nranks, bool gather);
void launch_tw_drift(const TrackParams& p, double half_len, cudaStream_t s);
// stage 1: first half drift, this rank's entries; stage 2 (after the gather): sort, scan, kick
// of this rank's particles, second half drift
void launch_transwake_sorted_stage(int stage, const TrackParams& p, const DevElem& e, const TwLayout& t,
                                   int rank, int64_t ntot_all, cudaStream_t s);
// the longitudinal wake in stages, for runs whose bunch is spread over several GPUs
struct LwParams { double half, energy, charge, Rs, fr, Q; int nbins; bool on; };
LwParams longwake_params(const DevElem& e_host);
void launch_longwake_stage(int stage, const TrackParams& p, const LwParams& w, double* scratch,
                           int32_t* counts, cudaStream_t s);
// scratch[0..5] from the exchanged z range and count (kern_coll.cu)
void launch_lw_regeom(double* scratch, int nbins, double charge_nc, cudaStream_t s);
// moments of live particles: out[0..5] mean, [6..11] sigma, [12..17] cross, [18] nlive.
// reduce (may be null) sums `count` device doubles over the ranks of a bunch spread over GPUs, in
// place on stream s, between the passes (the sums and count, then the centred moments); it
// returns a status, which the launcher returns (0: success)
typedef int (*StatReduce)(void* ctx, double* buf, int count, cudaStream_t s);
int launch_beam_stat(const double* st, int64_t n, double* partial, int nblk, double* out, cudaStream_t s,
                     StatReduce reduce = nullptr, void* rctx = nullptr);
int beam_stat_blocks(int64_t n);
double fp64_peak_run(int sm_count, cudaStream_t s, float* ms_out, double* sm_mhz_out);

// ---- plain (kern_plain.cu) ----------------------------------------------------------------
void launch_plain_elem(const TrackParams& p, int e, const int32_t* turn_ctr, cudaStream_t s);
void launch_plain_turn_end(const TrackParams& p, int32_t* turn_ctr, cudaStream_t s);
// exact mode: the plain kernel's arithmetic over [e0, e1) for nturn turns in one launch; with
// record, loss turns are recorded and the turn counter advanced by nturn (a second, tiny launch)
void launch_exact(const TrackParams& p, int e0, int e1, int nturn, int32_t* turn_ctr, bool record,
                  cudaStream_t s);
// exact tangent map (Dual<6>) / central differences through [e0, e1) of one table
// transfer matrix and its exact derivative in one knob (knob codes per element: kind * 16 + index)
void launch_m66_knob(const DevElem* tbl, int e0, int e1, const double* r0_dev, const int32_t* knob_dev,
                     double* m_dev, double* dm_dev, cudaStream_t s);
void launch_m66(const DevElem* tbl, int e0, int e1, const double* r0_dev, double delta, int method,
                double* m_dev, cudaStream_t s);

// ---- adjoint (kern_adjoint.cu) ------------------------------------------------------------
struct AdjParams {
    const DevElem* tbl;
    int ne;
    int64_t n;
    double* st;             // SoA state being advanced
    double* lam;            // SoA adjoint
    double* tape;           // [ne][6][n] element-input states of one turn
    double* pgrad_part;     // [nblocks][nparam] per-block parameter-gradient rows
    const int32_t* pfirst;  // [ne] first parameter of each element (sorted by element)
    const int32_t* pcount;  // [ne] parameters of each element
    const int32_t* pkind;   // [nparam] adj::ParamKind
    const int32_t* pindex;  // [nparam] multipole index
    int nparam;
    const int32_t* pelem;   // [npe] the parameter elements in line order
    const int32_t* unit_zd; // [npe + 1] 1 where a tape unit has an element that reads z or changes delta
};
int adj_blocks(int64_t n);
// turn_tape: null, or room for every turn's starting state (nturn x 6 x n doubles)
// turns [t0, t0 + nturn) of the run; st carries the state between consecutive launches
// threads: block size (64, 128 or 256); sm_fwd: null, or kAdjSmSlots counters of the forward
// blocks running on each SM (for a tape kernel running beside the forward)
constexpr int kAdjSmSlots = 256;
void launch_adj_forward(const AdjParams& a, double* ckpt, int t0, int nturn, int every, double* turn_tape,
                        cudaStream_t s, int threads = 64, int* sm_fwd = nullptr);
// turn-start states of checkpoint segments seg0 .. seg0+nseg-1 into turn_tape, from turn seg0 * every on
void launch_adj_recompute(const AdjParams& a, const double* ckpt, double* turn_tape, int nturn, int every,
                          int seg0, int nseg, cudaStream_t s);
void launch_adj_turn_reverse(const AdjParams& a, const double* r_start, const double* final_x, cudaStream_t s);
void launch_adj_reduce(const double* part, int nblk, int nparam, double* out, cudaStream_t s);
// block-Jacobian tape of nt turns (unit Jacobians and parameter sensitivities) and the reverse
// sweep over it (kern_adjoint.cu)
// general: the line has elements or parameters outside the explicit-Jacobian maps
// (jtape_needs_general)
// *flag = 1 when any of v[0 .. n) is non-zero (the launcher zeroes it first, on s)
void launch_any_nonzero(const double* v, int64_t n, int* flag, cudaStream_t s);
// work: null (one unit per thread), or a zeroed counter: a grid of the resident blocks takes
// groups of units from it, leaving the SMs sm_fwd marks (sm_count: the device's SMs).
// zrow = false: the z rows of units with no element that reads z are left at e_z (valid for a
// line with no such element swept with a seed whose z components are zero)
void launch_adj_jtape(const AdjParams& a, const double* turn_tape, int j0, int nt, const double* final_x,
                      int npe, double* jt, double* sens, bool general, cudaStream_t s, int* work = nullptr,
                      const int* sm_fwd = nullptr, int sm_count = 0, bool zrow = true);
bool jtape_needs_general(const DevElem* host_tbl, int ne, const int32_t* pcount, const int32_t* pfirst,
                         const int32_t* pkind);
// per tape unit (npe + 1 of them): 1 if any of its elements is not a drift, straight multipole,
// radiation-free bend, aperture or marker
void jtape_unit_zd(const DevElem* host_tbl, int ne, const int32_t* pelem, int npe, int32_t* unit_zd);
// grow: per-lane gradient rows in global memory, ntile x nparam x 32 doubles, used only past
// 384 parameters (null otherwise)
void launch_adj_jsweep(const AdjParams& a, int nt, const double* final_x, int npe, const int32_t* pelem,
                       const double* jt, const double* sens, double* grow, cudaStream_t s);
// rows of the per-block gradient partials (covers both the sweep's tiles and the reverse kernel's blocks)
int adj_part_rows(int64_t n);
// doubles of the tiled tapes per turn and unit (ceil(n / 32) * 32 particles)
inline int64_t adj_tile_span(int64_t n) { return (n + 31) / 32 * 32; }

}  // namespace accel
