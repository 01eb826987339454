// capi_adjoint.cpp — the forward/backward C-ABI pair of the adjoint.
//
// accel_adjoint_forward tracks N particles for nturn turns (literal maps, effective Horner order),
// keeping the state at every ckpt_every-th turn.  The reverse pass needs, per turn, the unit
// Jacobians (the 6x6 maps from one parameter element's output to the next one's) and the
// parameter sensitivities, taped by one wide kernel over (turn, particle), and one kernel per
// 32-particle tile sweeps them backwards (kern_adjoint.cu).  How they are scheduled depends on
// the tape budget (accel_set_adjoint_tape_budget; by default half of the free device memory):
//   whole run   every turn's Jacobians fit: the forward runs in launches of 32 turns and each
//               chunk is taped on a second stream as soon as the forward has written its turn
//               starts, so the taping (wide, FP64-bound) runs behind the forward (one particle
//               per thread, latency-bound); the forward's blocks mark their SMs and the tape
//               kernel's blocks leave those SMs, so the two share the GPU by SMs rather than
//               by issue slots; the backward is a single sweep over the run;
//   chunks      accel_adjoint_backward walks the segments last to first: the segment's turn
//               starts (kept by the forward when they fit, else recomputed from its checkpoint),
//               then, chunk by chunk, last to first, the tape and its sweep;
//   per turn    when not even one turn's tape fits, each turn is reversed element by element
//               (one launch per turn, an element-input tape of ne x 6 x N).
// Memory on the device: (nseg + K + 3) x 6 x N doubles for checkpoints, turn-start states, state,
// adjoint and scratch, plus the tape.
//
// Parameters are (element, field, index) triples: StrMPole PolynomB/PolynomA[index] (field K on a
// StrMPole is PolynomB[1]), Quad K.  The line must be free of radiation, quantum excitation and
// wake elements (their maps are not differentiated): ACCEL_E_UNSUPPORTED otherwise.
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>
#include "adjoint_params.h"
#include "engine.h"
#include "kernels.h"
#include "runtime.h"

using namespace accel;

#define CK(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(ACCEL_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

namespace {
constexpr int kMaxAdjParams = 2048;
// Device memory each tape may take (the turn starts; the Jacobians): accel_set_adjoint_tape_budget,
// or by default half of the device memory free when the adjoint is created, at least 4e9 bytes.
constexpr double kTapeBudgetFloor = 4.0e9;
std::atomic<double> g_tape_budget{-1.0};  // <= 0: the default
constexpr int kForwardChunk = 32;  // turns per forward launch when the tapes follow it chunk by chunk
// Forward block size in that mode: 4,096 particles take 32 SMs (one warp per scheduler, the
// forward's latency-bound chain at full speed) and the tape kernel leaves those SMs to it.
// Measured per gradient (4,096 particles, 512 turns, 36 knobs): 239 ms with 64-thread blocks
// and tape blocks anywhere; 192-204 ms like this; 16- and 64-turn chunks, 256-thread blocks, or
// one or two tape blocks left on each forward SM were slower (189-394 ms forward).
constexpr int kForwardThreads = 128;

double tape_budget() {
    const double b = g_tape_budget.load();
    if (b > 0) return b;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        fr = 0;
    }
    return std::max(kTapeBudgetFloor, 0.5 * (double)fr);
}

bool dev_ptr(const void* p) {
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}
}  // namespace

struct accel_adjoint {
    accel_line* line = nullptr;
    int n = 0, nturn = 0, every = 1, nseg = 0, ne = 0, nparam = 0;
    std::vector<int> order;  // caller's parameter j -> sorted position
    std::vector<int32_t> pfirst, pcount, pkind, pindex;
    std::vector<int32_t> pelem;  // elements carrying parameters, in line order
    int npe = 0;
    int chunk = 0;               // turns per block-Jacobian tape; 0: per-turn element reversal
    bool general = true;         // the tape needs the dual-number fallback (jtape_needs_general)
    // no element of the line reads z or changes delta (and the tape is the explicit one): a
    // reverse sweep seeded with zero z components never uses the unit Jacobians' z rows, so
    // the tapes are written without them, and a seed with a z component has them re-taped
    bool zrow_free = false;
    bool tapes_zrow = true;      // the whole-run tapes of the last forward carry the z rows
    DevBuf flag;
    bool all_turns = false;      // turn_tape holds every turn of the run, written by the forward
    // the Jacobian tape of every turn of the run fits the budget: the forward runs in chunks of
    // kForwardChunk turns and each chunk's tape is written on the second stream as soon as its
    // turn starts are out, behind the forward; the backward is then one sweep
    bool whole = false;
    cudaStream_t tape_stream = nullptr;
    cudaStream_t fwd_stream = nullptr;  // the forward's launches, at the device's highest priority
    cudaEvent_t fwd_ready = nullptr;    // the forward may start (after the caller's input copy)
    cudaEvent_t fwd_done = nullptr;
    std::vector<cudaEvent_t> chunk_ev;  // the forward has written chunk c's turn starts
    cudaEvent_t tape_done = nullptr;    // every tape of the last forward is written
    // whole-run mode: kAdjSmSlots counters of the forward blocks on each SM, then one work
    // counter per chunk's tape (zeroed at the start of each forward)
    DevBuf sched;
    DevBuf st, lam, aos, tape, ckpt, turn_tape, part, meta, final_x, grad, jt, rt, pel, grow, uzd;
    bool have_forward = false;
    ~accel_adjoint() {
        if (tape_stream) cudaStreamSynchronize(tape_stream);
        if (fwd_stream) cudaStreamSynchronize(fwd_stream);
        for (cudaEvent_t e : chunk_ev) cudaEventDestroy(e);
        for (cudaEvent_t e : {tape_done, fwd_ready, fwd_done})
            if (e) cudaEventDestroy(e);
        if (tape_stream) cudaStreamDestroy(tape_stream);
        if (fwd_stream) cudaStreamDestroy(fwd_stream);
        for (DevBuf* b : {&st, &lam, &aos, &tape, &ckpt, &turn_tape, &part, &meta, &final_x, &grad, &jt, &rt, &pel,
                          &grow, &uzd, &sched, &flag})
            b->release();
    }
};

static AdjParams params_of(accel_adjoint* J) {
    AdjParams a{};
    a.tbl = (const DevElem*)J->line->d_tbl.p;
    a.ne = J->ne;
    a.n = J->n;
    a.st = (double*)J->st.p;
    a.lam = (double*)J->lam.p;
    a.tape = (double*)J->tape.p;
    a.pgrad_part = (double*)J->part.p;
    int32_t* m = (int32_t*)J->meta.p;
    a.pfirst = m;
    a.pcount = m + J->ne;
    a.pkind = m + 2 * J->ne;
    a.pindex = m + 2 * J->ne + std::max(1, J->nparam);
    a.nparam = J->nparam;
    a.pelem = (const int32_t*)J->pel.p;
    a.unit_zd = (const int32_t*)J->uzd.p;
    return a;
}

extern "C" {

int accel_set_adjoint_tape_budget(int64_t bytes) {
    g_tape_budget = bytes <= 0 ? -1.0 : (double)bytes;
    return ACCEL_OK;
}

int accel_adjoint_create(accel_line* L, int N, int nturn, int every, const int32_t* pe,
                         const int32_t* pf, const int32_t* pi, int nparam, accel_adjoint** out) {
    if (!L || !out || N <= 0 || nturn <= 0 || every <= 0 || nparam < 0) return fail(ACCEL_E_INVALID, "bad argument");
    if (nparam > 0 && (!pe || !pf || !pi)) return fail(ACCEL_E_INVALID, "parameter arrays are NULL");
    if (nparam > kMaxAdjParams) return fail(ACCEL_E_TOO_LARGE, "more than 2048 parameters");
    accel_ctx* C = L->ctx;
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    int s = line_sync(L);
    if (s) return s;
    const int ne = (int)L->desc.size();
    for (int k = 0; k < ne; k++) {
        const accel_elem_desc& d = L->desc[k];
        if (!is_supported(d.type)) return fail(ACCEL_E_UNSUPPORTED, std::string("element ") + d.famname + " is not implemented");
        if (is_collective(d.type)) return fail(ACCEL_E_UNSUPPORTED, "the adjoint does not differentiate wake elements");
        if (d.type == ACCEL_BENDMPOLE && d.flags != 0) return fail(ACCEL_E_UNSUPPORTED, "the adjoint needs radiation off");
        if (d.type == ACCEL_SYNCRAD && d.flags != 0) return fail(ACCEL_E_UNSUPPORTED, "the adjoint needs SyncRad off");
        if ((d.type == ACCEL_CRABCAV && d.flags != 0 && (d.f[5] > 0 || d.f[6] > 0)) ||
            (d.type == ACCEL_RFMULT && d.f[3] > 0))
            return fail(ACCEL_E_UNSUPPORTED, "the adjoint needs RF phase and voltage noise off");
    }
    std::unique_ptr<accel_adjoint> J(new accel_adjoint());
    J->line = L;
    J->n = N;
    J->nturn = nturn;
    J->every = every;
    J->nseg = (nturn + every - 1) / every;
    J->ne = ne;
    J->nparam = nparam;
    // parameters, stably sorted by element
    struct P { int elem, kind, index, orig; };
    std::vector<P> ps;
    for (int j = 0; j < nparam; j++) {
        const int e = pe[j];
        if (e < 0 || e >= ne) return fail(ACCEL_E_INVALID, "parameter element out of range");
        const accel_elem_desc& d = L->desc[e];
        P p{e, 0, pi[j], j};
        if (d.type == ACCEL_STRMPOLE && (pf[j] == ACCEL_F_POLYNOMB || pf[j] == ACCEL_F_POLYNOMA)) {
            if (pi[j] < 0 || pi[j] >= ACCEL_MAX_MPOLE) return fail(ACCEL_E_INVALID, "multipole index outside 0..9");
            p.kind = pf[j] == ACCEL_F_POLYNOMB ? adj::PK_B : adj::PK_A;
        } else if (d.type == ACCEL_STRMPOLE && pf[j] == ACCEL_F_K) {
            p.kind = adj::PK_B;
            p.index = 1;
        } else if (d.type == ACCEL_QUAD && pf[j] == ACCEL_F_K) {
            p.kind = adj::PK_QUADK;
            p.index = 0;
        } else {
            return fail(ACCEL_E_UNSUPPORTED, std::string("no gradient for this field of ") + d.famname);
        }
        ps.push_back(p);
    }
    std::stable_sort(ps.begin(), ps.end(), [](const P& a, const P& b) { return a.elem < b.elem; });
    J->order.assign((size_t)nparam, 0);
    J->pfirst.assign((size_t)ne, 0);
    J->pcount.assign((size_t)ne, 0);
    for (int j = 0; j < nparam; j++) {
        J->order[(size_t)ps[(size_t)j].orig] = j;
        J->pkind.push_back(ps[(size_t)j].kind);
        J->pindex.push_back(ps[(size_t)j].index);
        J->pcount[(size_t)ps[(size_t)j].elem]++;
    }
    for (int e = 0, acc = 0; e < ne; e++) {
        J->pfirst[(size_t)e] = acc;
        acc += J->pcount[(size_t)e];
        if (J->pcount[(size_t)e] > adj::kMaxParamsPerElem)
            return fail(ACCEL_E_TOO_LARGE, "more than 4 parameters on one element");
    }
    // a StrMPole parameter beyond the element's effective order still needs its Horner terms:
    // the gradient of B_n at a zero coefficient is the derivative of the zero term
    for (const P& p : ps) {
        if (p.kind == adj::PK_QUADK) continue;
        DevElem& r = L->host_tbl[(size_t)p.elem];
        if (p.index > r.order_eff) {
            r.order_eff = (int8_t)p.index;
            if (p.kind == adj::PK_A) r.flags |= STR_SKEW, r.flags &= ~STR_SKEW0;
        }
    }
    CK(cudaMemcpy(L->d_tbl.p, L->host_tbl.data(), L->host_tbl.size() * sizeof(DevElem), cudaMemcpyHostToDevice));
    const size_t s6 = sizeof(double) * 6 * (size_t)N;
    const int nblk = adj_part_rows(N);
    for (int e = 0; e < ne; e++)
        if (J->pcount[(size_t)e] > 0) J->pelem.push_back(e);
    J->npe = (int)J->pelem.size();
    J->general = jtape_needs_general(L->host_tbl.data(), ne, J->pcount.data(), J->pfirst.data(), J->pkind.data());
    // every turn-start state kept by the forward when that fits the tape budget: the reverse
    // pass then recomputes nothing (otherwise each segment is recomputed from its checkpoint)
    const double budget = tape_budget();
    J->all_turns = (double)s6 * nturn <= budget;
    const size_t span = (size_t)adj_tile_span(N);  // tiled tapes: 32-particle tiles
    const double per_turn = 8.0 * (double)span * (36.0 * (J->npe + 1) + 6.0 * nparam);
    J->chunk = (int)std::min<double>(std::min(every, nturn), std::floor(budget / per_turn));
    J->whole = J->all_turns && per_turn * nturn <= budget;
    if (J->chunk >= 1) {
        const size_t c = (size_t)(J->whole ? nturn : J->chunk), nn = span;
        if ((s = J->jt.ensure(sizeof(double) * c * (size_t)(J->npe + 1) * 36 * nn)) ||
            (s = J->rt.ensure(sizeof(double) * std::max<size_t>(1, c * (size_t)nparam * 6 * nn))) ||
            (nparam > 384 && (s = J->grow.ensure(sizeof(double) * nn * (size_t)nparam))) ||
            (s = J->pel.ensure(sizeof(int32_t) * (size_t)std::max(1, J->npe))) ||
            (s = J->uzd.ensure(sizeof(int32_t) * (size_t)(J->npe + 1))))
            return s;
        if (J->npe > 0)
            CK(cudaMemcpy(J->pel.p, J->pelem.data(), sizeof(int32_t) * J->pelem.size(), cudaMemcpyHostToDevice));
        std::vector<int32_t> uz((size_t)J->npe + 1);
        jtape_unit_zd(L->host_tbl.data(), ne, J->pelem.data(), J->npe, uz.data());
        CK(cudaMemcpy(J->uzd.p, uz.data(), sizeof(int32_t) * uz.size(), cudaMemcpyHostToDevice));
        J->zrow_free = !J->general && std::all_of(uz.begin(), uz.end(), [](int32_t z) { return z == 0; });
        if ((s = J->flag.ensure(sizeof(int)))) return s;
        if (J->whole) {
            // the forward on the highest-priority stream: a chunk's blocks are placed ahead of
            // the tape blocks waiting for room, so the latency-bound forward is not held back
            int least = 0, greatest = 0;
            CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
            CK(cudaStreamCreateWithPriority(&J->fwd_stream, cudaStreamNonBlocking, greatest));
            CK(cudaStreamCreateWithPriority(&J->tape_stream, cudaStreamNonBlocking, least));
            CK(cudaEventCreateWithFlags(&J->fwd_ready, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&J->fwd_done, cudaEventDisableTiming));
            J->chunk_ev.assign((size_t)((nturn + kForwardChunk - 1) / kForwardChunk), nullptr);
            for (cudaEvent_t& e : J->chunk_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&J->tape_done, cudaEventDisableTiming));
            if ((s = J->sched.ensure(sizeof(int) * (kAdjSmSlots + J->chunk_ev.size())))) return s;
        }
    } else {
        J->chunk = 0;
        if ((s = J->tape.ensure(s6 * (size_t)ne))) return s;
    }
    if ((s = J->st.ensure(s6)) || (s = J->lam.ensure(s6)) || (s = J->aos.ensure(s6)) ||
        (s = J->ckpt.ensure(s6 * (size_t)J->nseg)) ||
        (s = J->turn_tape.ensure(s6 * (size_t)(J->all_turns ? nturn : std::min(every, nturn)))) ||
        (s = J->part.ensure(sizeof(double) * (size_t)std::max(1, nblk * nparam))) ||
        (s = J->meta.ensure(sizeof(int32_t) * (size_t)(2 * ne + 2 * std::max(1, nparam)))) ||
        (s = J->final_x.ensure(sizeof(double) * (size_t)N)) ||
        (s = J->grad.ensure(sizeof(double) * (size_t)std::max(1, nparam))))
        return s;
    std::vector<int32_t> meta((size_t)(2 * ne + 2 * std::max(1, nparam)), 0);
    std::copy(J->pfirst.begin(), J->pfirst.end(), meta.begin());
    std::copy(J->pcount.begin(), J->pcount.end(), meta.begin() + ne);
    std::copy(J->pkind.begin(), J->pkind.end(), meta.begin() + 2 * ne);
    std::copy(J->pindex.begin(), J->pindex.end(), meta.begin() + 2 * ne + std::max(1, nparam));
    CK(cudaMemcpy(J->meta.p, meta.data(), meta.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    L->refs.fetch_add(1);
    *out = J.release();
    return ACCEL_OK;
}

int accel_adjoint_destroy(accel_adjoint* J) {
    if (!J) return ACCEL_OK;
    accel_line* L = J->line;
    {
        std::lock_guard<std::mutex> lk(L->ctx->mu);
        cudaSetDevice(L->ctx->device);
        cudaStreamSynchronize(L->ctx->stream);
        L->dirty = true;  // the table was widened for parameter orders; rebuild on next use
        delete J;
    }
    accel::line_unref(L);
    return ACCEL_OK;
}

int accel_adjoint_forward(accel_adjoint* J, const double* r0, double* r_final) {
    if (!J || !r0 || !r_final) return fail(ACCEL_E_INVALID, "NULL argument");
    accel_ctx* C = J->line->ctx;
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    if (J->line->dirty) return fail(ACCEL_E_INVALID, "the line changed after accel_adjoint_create");
    cudaStream_t s = C->stream;
    const size_t s6 = sizeof(double) * 6 * (size_t)J->n;
    const double* in = r0;
    if (!dev_ptr(r0)) {
        CK(cudaMemcpyAsync(J->aos.p, r0, s6, cudaMemcpyHostToDevice, s));
        in = (const double*)J->aos.p;
    }
    launch_aos_to_soa(in, (double*)J->st.p, J->n, s);
    AdjParams a = params_of(J);
    if (J->whole) {
        // forward in chunks; each chunk's Jacobian tape on the second stream as soon as the
        // chunk's turn starts are written, so the taping runs behind the forward
        const size_t span = (size_t)adj_tile_span(J->n);
        double* jt = (double*)J->jt.p;
        double* rt = (double*)J->rt.p;
        int c = 0;
        int* sm_fwd = (int*)J->sched.p;
        int* work = sm_fwd + kAdjSmSlots;
        CK(cudaMemsetAsync(J->sched.p, 0, sizeof(int) * (kAdjSmSlots + J->chunk_ev.size()), s));
        CK(cudaEventRecord(J->fwd_ready, s));
        CK(cudaStreamWaitEvent(J->fwd_stream, J->fwd_ready, 0));
        CK(cudaStreamWaitEvent(J->tape_stream, J->fwd_ready, 0));
        for (int t0 = 0; t0 < J->nturn; t0 += kForwardChunk, c++) {
            const int nt = std::min(kForwardChunk, J->nturn - t0);
            launch_adj_forward(a, (double*)J->ckpt.p, t0, nt, J->every, (double*)J->turn_tape.p, J->fwd_stream,
                               kForwardThreads, sm_fwd);
            CK(cudaEventRecord(J->chunk_ev[(size_t)c], J->fwd_stream));
            CK(cudaStreamWaitEvent(J->tape_stream, J->chunk_ev[(size_t)c], 0));
            launch_adj_jtape(a, (const double*)J->turn_tape.p, t0, nt, nullptr, J->npe,
                             jt + (size_t)t0 * (J->npe + 1) * 36 * span, rt + (size_t)t0 * J->nparam * 6 * span,
                             J->general, J->tape_stream, work + c, sm_fwd, C->sm_count, !J->zrow_free);
        }
        J->tapes_zrow = !J->zrow_free;
        CK(cudaEventRecord(J->fwd_done, J->fwd_stream));
        CK(cudaEventRecord(J->tape_done, J->tape_stream));
        CK(cudaStreamWaitEvent(s, J->fwd_done, 0));
        CK(cudaStreamWaitEvent(s, J->tape_done, 0));  // the call returns with the tapes written
        C->launches += 2 * c;
    } else {
        launch_adj_forward(a, (double*)J->ckpt.p, 0, J->nturn, J->every,
                           J->all_turns ? (double*)J->turn_tape.p : nullptr, s);
        C->launches += 1;
    }
    CK(cudaMemcpyAsync(J->final_x.p, J->st.p, sizeof(double) * (size_t)J->n, cudaMemcpyDeviceToDevice, s));
    launch_soa_to_aos((const double*)J->st.p, (double*)J->aos.p, J->n, s);
    C->launches += 2;
    if (dev_ptr(r_final)) CK(cudaMemcpyAsync(r_final, J->aos.p, s6, cudaMemcpyDeviceToDevice, s));
    else CK(cudaMemcpyAsync(r_final, J->aos.p, s6, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    CK(cudaGetLastError());
    J->have_forward = true;
    return ACCEL_OK;
}

int accel_adjoint_backward(accel_adjoint* J, const double* g, double* dr0, double* dp) {
    if (!J || !g || !dr0 || (!dp && J->nparam > 0)) return fail(ACCEL_E_INVALID, "NULL argument");
    if (!J->have_forward) return fail(ACCEL_E_INVALID, "call accel_adjoint_forward first");
    accel_ctx* C = J->line->ctx;
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    cudaStream_t s = C->stream;
    const size_t s6 = sizeof(double) * 6 * (size_t)J->n;
    const double* in = g;
    if (!dev_ptr(g)) {
        CK(cudaMemcpyAsync(J->aos.p, g, s6, cudaMemcpyHostToDevice, s));
        in = (const double*)J->aos.p;
    }
    launch_aos_to_soa(in, (double*)J->lam.p, J->n, s);
    const int nblk = adj_part_rows(J->n);
    if (J->nparam > 0) CK(cudaMemsetAsync(J->part.p, 0, sizeof(double) * (size_t)nblk * J->nparam, s));
    AdjParams a = params_of(J);
    int64_t launches = 1;
    // z rows are needed when the seed has a z component (or the line reads z)
    bool zrow = !J->zrow_free;
    if (!zrow && J->chunk > 0) {
        int any = 0;
        launch_any_nonzero((const double*)J->lam.p + 4 * (size_t)J->n, J->n, (int*)J->flag.p, s);
        CK(cudaMemcpyAsync(&any, J->flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        zrow = any != 0;
        launches++;
    }
    // the forward wrote every turn's tape, without z rows: a seed with a z component has them
    // written again, with z rows, from the kept turn starts
    if (J->whole && zrow && !J->tapes_zrow) {
        const size_t span = (size_t)adj_tile_span(J->n);
        for (int t0 = 0; t0 < J->nturn; t0 += kForwardChunk) {
            const int nt = std::min(kForwardChunk, J->nturn - t0);
            launch_adj_jtape(a, (const double*)J->turn_tape.p, t0, nt, (const double*)J->final_x.p, J->npe,
                             (double*)J->jt.p + (size_t)t0 * (J->npe + 1) * 36 * span,
                             (double*)J->rt.p + (size_t)t0 * J->nparam * 6 * span, J->general, s);
            launches++;
        }
        J->tapes_zrow = true;
    }
    // the forward wrote every turn's tape: one sweep over the whole run, last turn to first
    if (J->whole) {
        launch_adj_jsweep(a, J->nturn, (const double*)J->final_x.p, J->npe, (const int32_t*)J->pel.p,
                          (const double*)J->jt.p, (const double*)J->rt.p, (double*)J->grow.p, s);
        launches++;
    }
    // with all_turns the forward kept every turn's starting state: nothing to recompute
    for (int seg = J->whole ? -1 : J->nseg - 1; seg >= 0; seg--) {
        const int t0 = seg * J->every;
        const int nt = std::min(J->every, J->nturn - t0);
        const double* tt = (const double*)J->turn_tape.p;  // this segment's turn-start states
        if (J->all_turns) {
            tt += (size_t)t0 * 6 * J->n;
        } else {
            launch_adj_recompute(a, (const double*)J->ckpt.p, (double*)J->turn_tape.p, J->nturn, J->every, seg, 1, s);
            launches++;
        }
        if (J->chunk > 0) {
            for (int hi = nt; hi > 0; hi -= J->chunk) {
                const int lo = std::max(0, hi - J->chunk);
                launch_adj_jtape(a, tt, lo, hi - lo, (const double*)J->final_x.p, J->npe, (double*)J->jt.p,
                                 (double*)J->rt.p, J->general, s, nullptr, nullptr, 0, zrow);
                launch_adj_jsweep(a, hi - lo, (const double*)J->final_x.p, J->npe, (const int32_t*)J->pel.p,
                                  (const double*)J->jt.p, (const double*)J->rt.p, (double*)J->grow.p, s);
                launches += 2;
            }
        } else {
            for (int j = nt - 1; j >= 0; j--) {
                launch_adj_turn_reverse(a, tt + (size_t)j * 6 * J->n, (const double*)J->final_x.p, s);
                launches++;
            }
        }
    }
    launch_soa_to_aos((const double*)J->lam.p, (double*)J->aos.p, J->n, s);
    launches++;
    if (dev_ptr(dr0)) CK(cudaMemcpyAsync(dr0, J->aos.p, s6, cudaMemcpyDeviceToDevice, s));
    else CK(cudaMemcpyAsync(dr0, J->aos.p, s6, cudaMemcpyDeviceToHost, s));
    if (J->nparam > 0) {
        launch_adj_reduce((const double*)J->part.p, nblk, J->nparam, (double*)J->grad.p, s);
        launches++;
        std::vector<double> sorted((size_t)J->nparam);
        CK(cudaMemcpyAsync(sorted.data(), J->grad.p, sizeof(double) * J->nparam, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        std::vector<double> outv((size_t)J->nparam);
        for (int j = 0; j < J->nparam; j++) outv[(size_t)j] = sorted[(size_t)J->order[(size_t)j]];
        if (dev_ptr(dp)) CK(cudaMemcpy(dp, outv.data(), sizeof(double) * J->nparam, cudaMemcpyHostToDevice));
        else std::memcpy(dp, outv.data(), sizeof(double) * J->nparam);
    }
    CK(cudaStreamSynchronize(s));
    CK(cudaGetLastError());
    C->launches += launches;
    return ACCEL_OK;
}

}  // extern "C"
