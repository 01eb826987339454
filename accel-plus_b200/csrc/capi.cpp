// capi.cpp — the C-ABI: contexts, lines, tracking orchestration, autotuning.
//
// A tracking request becomes a sequence of kernel launches captured into one CUDA graph:
//   fused mode:  init live list | { fused segment of K turns | stable compaction } x ceil(T/K)
//                (rings with a wake element run one turn per segment, split at the wake)
//   plain mode:  one graph per turn: one launch per element, then the per-turn loss scan,
//                replayed T times.
// Graphs are cached per request shape, so repeated identical calls (a benchmark loop, a DA scan
// over many grids of the same size) relaunch without host-side rebuilding.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>
#include <dlfcn.h>
#include <nccl.h>
#include "engine.h"
#include "kernels.h"
#include "runtime.h"

using namespace accel;

namespace accel {
thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int status, const std::string& msg) {
    set_error(msg);
    return status;
}
}  // namespace accel

#define CK(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(ACCEL_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

// ------------------------------------------------------------------------------------------
// device buffers
// ------------------------------------------------------------------------------------------
// bytes of device memory held in DevBufs, and the budget (accel_set_device_memory_limit)
static std::atomic<int64_t> g_held{0};
static std::atomic<int64_t> g_limit{-1};

int DevBuf::ensure(size_t nbytes) {
    if (nbytes <= bytes && p) return ACCEL_OK;
    size_t want = std::max<size_t>(nbytes, 256);
    const int64_t limit = g_limit.load();
    if (limit >= 0 && g_held.load() - (int64_t)bytes + (int64_t)want > limit)
        return fail(ACCEL_E_NOMEM, "a device buffer of " + std::to_string(want) + " bytes would take the library's " +
                                       "device memory above its limit of " + std::to_string(limit) + " bytes");
    release();
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        return fail(ACCEL_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    bytes = want;
    g_held += (int64_t)want;
    return ACCEL_OK;
}
void DevBuf::release() {
    if (p) {
        cudaFree(p);
        g_held -= (int64_t)bytes;
    }
    p = nullptr;
    bytes = 0;
}

extern "C" int accel_set_device_memory_limit(int64_t bytes) {
    g_limit = bytes < 0 ? -1 : bytes;
    return ACCEL_OK;
}

extern "C" int accel_device_memory_held(int64_t* bytes) {
    if (!bytes) return fail(ACCEL_E_INVALID, "NULL argument");
    *bytes = g_held.load();
    return ACCEL_OK;
}

static bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

accel_ctx::~accel_ctx() {
    cudaSetDevice(device);
    graphs.clear();
    for (DevBuf* b : {&state, &aos, &loss, &live0, &cnt, &tables, &tbl_off, &pinst, &scratch,
                      &iscratch, &probe_state, &tw_scratch, &hot})
        b->release();
    for (cudaEvent_t e : prof_events) cudaEventDestroy(e);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
}

GraphEntry::~GraphEntry() {
    for (cudaGraphExec_t e : exec)
        if (e) cudaGraphExecDestroy(e);
}

// ------------------------------------------------------------------------------------------
// line compilation
// ------------------------------------------------------------------------------------------
int accel::line_sync(accel_line* L) {
    if (!L->dirty && L->d_tbl.p) return ACCEL_OK;
    std::vector<DevElem> recs;
    std::string err;
    int s = compile_line(L->desc.data(), (int)L->desc.size(), recs, err);
    if (s != ACCEL_OK) return fail(s, err);
    cudaSetDevice(L->ctx->device);
    // WigTable kick tables: one device block per line, each record given its table's address
    std::vector<double> aux;
    std::vector<std::pair<size_t, size_t>> at;  // (record, offset in doubles)
    for (size_t k = 0; k < recs.size(); k++) {
        if (recs[k].op != OP_WIGTABLE) continue;
        auto t = wigtable_find((int32_t)recs[k].v[V_TID]);
        if (!t) return fail(ACCEL_E_INVALID, "WigTable kick table was destroyed");
        at.push_back({k, aux.size()});
        aux.insert(aux.end(), t->data.begin(), t->data.end());
    }
    int st = 0;
    if (!aux.empty()) {
        st = L->d_aux.ensure(aux.size() * sizeof(double));
        if (st) return st;
        CK(cudaMemcpy(L->d_aux.p, aux.data(), aux.size() * sizeof(double), cudaMemcpyHostToDevice));
        for (auto& a : at) {
            const double* dp = (const double*)L->d_aux.p + a.second;
            static_assert(sizeof(dp) == sizeof(double), "a device address must fit a payload slot");
            std::memcpy(&recs[a.first].v[V_TPTR], &dp, sizeof(dp));
        }
    }
    L->host_tbl = recs;
    st = L->d_tbl.ensure(std::max<size_t>(1, recs.size()) * sizeof(DevElem));
    if (st) return st;
    if (!recs.empty())
        CK(cudaMemcpy(L->d_tbl.p, recs.data(), recs.size() * sizeof(DevElem), cudaMemcpyHostToDevice));
    if (!L->d_rng.p) {
        st = L->d_rng.ensure(sizeof(int32_t) * 2);
        if (st) return st;
        CK(cudaMemset(L->d_rng.p, 0, sizeof(int32_t) * 2));
    }
    L->dirty = false;
    L->version++;
    return ACCEL_OK;
}

static int check_supported(const accel_line* L, int e0, int e1) {
    for (int k = e0; k < e1; k++)
        if (!is_supported(L->desc[k].type))
            return fail(ACCEL_E_UNSUPPORTED, std::string("element ") + std::to_string(k) + " (" +
                                                 L->desc[k].famname + ", type " +
                                                 type_name(L->desc[k].type) +
                                                 ") is not implemented on the device");
    return ACCEL_OK;
}

// ------------------------------------------------------------------------------------------
// the core: track SoA device state for `nturn` turns through [e0, e1)
// ------------------------------------------------------------------------------------------
// ---- NCCL, loaded at run time ----------------------------------------------------------------
// The library links no NCCL; a context that is given a communicator (accel_ctx_set_comm) loads
// libnccl.so.2 and resolves the six functions it uses.
struct NcclApi {
    bool ok = false;
    std::string err;
    ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t) = nullptr;
    ncclResult_t (*AllGather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
    const char* (*GetErrorString)(ncclResult_t) = nullptr;
};

static NcclApi& nccl() {
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_LOCAL);
        if (!h) { api.err = std::string("cannot load libnccl.so.2: ") + dlerror(); return; }
        api.GetUniqueId = (decltype(api.GetUniqueId))dlsym(h, "ncclGetUniqueId");
        api.CommInitRank = (decltype(api.CommInitRank))dlsym(h, "ncclCommInitRank");
        api.CommDestroy = (decltype(api.CommDestroy))dlsym(h, "ncclCommDestroy");
        api.AllReduce = (decltype(api.AllReduce))dlsym(h, "ncclAllReduce");
        api.AllGather = (decltype(api.AllGather))dlsym(h, "ncclAllGather");
        api.GetErrorString = (decltype(api.GetErrorString))dlsym(h, "ncclGetErrorString");
        api.ok = api.GetUniqueId && api.CommInitRank && api.CommDestroy && api.AllReduce && api.AllGather &&
                 api.GetErrorString;
        if (!api.ok) api.err = "libnccl.so.2 lacks a required function";
    });
    return api;
}

static int nccl_fail(const char* what, ncclResult_t r) {
    return fail(ACCEL_E_CUDA, std::string(what) + ": " + nccl().GetErrorString(r));
}

struct CoreReq {
    accel_line* const* lines;
    int ninst;
    const DevElem* tables;
    const int32_t* tbl_off;
    const int32_t* pinst;
    double* st;
    int64_t ntot;
    int32_t* loss;
    int e0, e1, nturn, mode;
    int variant, seg, sched;
    bool probe;  // autotuning probe: no RNG advance bookkeeping
    int grid_staged;  // staged schedule: resident blocks on the device
    int64_t nrec;     // staged schedule: records in `tables` (instances x elements)
};

// A request is issued as four parts, each a short kernel sequence:
//   pre   initialise the live list, loss turns and the device turn counter
//   body  one segment: fused kernel for `seg` turns (or one turn of element launches in plain
//         mode, or one turn of local ranges and wake kernels), then the in-place compaction,
//         which also advances the turn counter; replayed nbody times
//   tail  the remaining turns when seg does not divide nturn
//   post  advance the line's QE turn base
// In graph mode each part is captured once into a CUDA graph (cached per request shape); in
// profiling mode the parts are issued directly with CUDA events around every fused launch.
enum Part { PART_PRE = 0, PART_BODY = 1, PART_TAIL = 2, PART_POST = 3 };

struct Plan {
    int seg = 1;      // turns per body
    int nbody = 0;    // body repetitions
    int tail = 0;     // turns in the tail (0: none)
};

// Fixed scratch size (doubles): wake bins and partials, beam-moment partials, m66 staging.  Kept
// constant so graphs that captured the scratch pointer never see it reallocated.
constexpr size_t kScratchDoubles = 65536;

constexpr int kExactSegTurns = 16;  // turns per exact-mode launch (a line without wakes)

static Plan make_plan(const CoreReq& q, bool has_coll) {
    Plan p;
    if (q.mode == ACCEL_MODE_FUSED && !has_coll) p.seg = std::max(1, std::min(q.seg, q.nturn));
    else if (q.mode == ACCEL_MODE_EXACT && !has_coll) p.seg = std::max(1, std::min(kExactSegTurns, q.nturn));
    else p.seg = 1;
    p.nbody = q.nturn / p.seg;
    p.tail = q.nturn - p.nbody * p.seg;
    return p;
}

static bool has_collective(const accel_line* L, int e0, int e1) {
    for (int k = e0; k < e1; k++)
        if (is_collective(L->desc[k].type)) return true;
    return false;
}

// Issue one part on stream s.  `mark` brackets each tracking-kernel launch (profiling).
template <class Mark>
static int emit_part(accel_ctx* C, const CoreReq& q, int part, int turns, cudaStream_t s,
                     Mark mark, int& launches) {
    accel_line* L0 = q.lines[0];
    int32_t* cnt = (int32_t*)C->cnt.p;  // [0] nlive [2] chunk [3] turn [4] err [5] lost since compaction
    int32_t* live = (int32_t*)C->live0.p;
    TrackParams P{};
    P.tables = q.tables;
    P.tbl_off = q.tbl_off;
    P.pinst = q.pinst;
    P.st = q.st;
    P.ntot = q.ntot;
    P.loss_turn = q.loss;
    P.live = live;
    P.nlive = cnt + 0;
    P.chunk_ctr = cnt + 2;
    P.turn_dev = cnt + 3;
    P.err = cnt + 4;
    P.lost_flag = cnt + 5;
    P.tw_pair_passes = cnt + 6;
    P.stage_wait = C->stage_wait;
    P.seed = L0->seed;
    P.rng_base = (int32_t*)L0->d_rng.p;
    P.turn0 = 0;
    P.rng_turn0 = 0;
    P.sched = q.sched;
    if (part == PART_PRE) {
        launch_init_live(q.st, q.ntot, q.loss, live, cnt + 0, cnt + 2, 1, s);
        launch_fill_i32(cnt + 3, 0, 3, s);  // turn counter, error word, lost flag
        launches += 2;
        if (q.mode == ACCEL_MODE_FUSED && q.sched == kSchedStaged) {
            launch_extract_hot(q.tables, q.nrec, C->hot.p, s);  // the lines the blocks stage
            launches++;
        }
        return ACCEL_OK;
    }
    if (part == PART_POST) {
        if (!q.probe) {
            launch_rng_advance((int32_t*)L0->d_rng.p, q.nturn, s);
            launches++;
        }
        return ACCEL_OK;
    }
    if (turns <= 0) return ACCEL_OK;
    int coll_status = ACCEL_OK;
    auto coll = [&](int k) {
        if (L0->desc[k].type == ACCEL_LONGWAKE) {
            double* scr = (double*)C->scratch.p;
            int32_t* counts = (int32_t*)C->iscratch.p;
            if (!C->comm) {
                launch_longwake(P, q.tables + k, L0->host_tbl[k], scr, counts, s);
                launches += L0->host_tbl[k].flags ? 5 : 2;
                return;
            }
            // the bunch is spread over the communicator's ranks: exchange its z range and live
            // count, then its bin counts (every rank takes the same steps: same lattice)
            const LwParams w = longwake_params(L0->host_tbl[k]);
            ncclComm_t cm = (ncclComm_t)C->comm;
            launch_longwake_stage(1, P, w, scr, counts, s);
            launches += 2;
            if (!w.on) return;
            ncclResult_t r = nccl().AllReduce(scr + 0, scr + 0, 1, ncclFloat64, ncclMin, cm, s);
            if (r == ncclSuccess) r = nccl().AllReduce(scr + 1, scr + 1, 1, ncclFloat64, ncclMax, cm, s);
            if (r == ncclSuccess) r = nccl().AllReduce(scr + 4, scr + 4, 1, ncclFloat64, ncclSum, cm, s);
            launch_lw_regeom(scr, w.nbins, w.charge, s);
            launch_longwake_stage(2, P, w, scr, counts, s);
            if (r == ncclSuccess) r = nccl().AllReduce(counts, counts, (size_t)w.nbins, ncclInt32, ncclSum, cm, s);
            launch_longwake_stage(3, P, w, scr, counts, s);
            launches += 4;
            if (r != ncclSuccess && coll_status == ACCEL_OK) coll_status = nccl_fail("ncclAllReduce (wake)", r);
        } else if (q.mode == ACCEL_MODE_FUSED) {
            // fused mode: the O(N log N) sum (kern_tw.cu), over all ranks' particles when a
            // communicator is set; plain and exact keep the pair sum
            const DevElem& e = L0->host_tbl[k];
            const bool gather = C->comm != nullptr;
            const TwLayout t = tw_layout(C->tw_scratch.p, C->tw_slots, gather ? C->nranks : 1, gather);
            launch_transwake_sorted_stage(1, P, e, t, gather ? C->rank : 0, C->tw_ntot_all, s);
            if (gather && e.flags) {
                ncclComm_t cm = (ncclComm_t)C->comm;
                const size_t m = (size_t)t.slots;
                ncclResult_t r = nccl().AllGather(t.key_s, t.key_g, m, ncclFloat64, cm, s);
                if (r == ncclSuccess) r = nccl().AllGather(t.x_s, t.x_g, m, ncclFloat64, cm, s);
                if (r == ncclSuccess) r = nccl().AllGather(t.y_s, t.y_g, m, ncclFloat64, cm, s);
                if (r == ncclSuccess) r = nccl().AllReduce(t.nvalid, t.nvalid + 1, 1, ncclInt32, ncclSum, cm, s);
                if (r != ncclSuccess && coll_status == ACCEL_OK) coll_status = nccl_fail("nccl (transverse wake)", r);
            }
            launch_transwake_sorted_stage(2, P, e, t, gather ? C->rank : 0, C->tw_ntot_all, s);
            // this library's kernels (the radix sort's are CUB's, not counted)
            launches += (e.flags ? 6 : 0) + (e.v[V_LEN] != 0 ? 2 : 0);
        } else {
            launch_transwake(P, q.tables + k, L0->host_tbl[k], nullptr, s);
            launches += 3;
        }
    };
    if (q.mode == ACCEL_MODE_FUSED) {
        const int grid = q.sched == kSchedStaged ? q.grid_staged : C->sm_count * std::max(1, C->bps[q.variant]);
        if (!has_collective(L0, q.e0, q.e1)) {
            P.e0 = q.e0;
            P.e1 = q.e1;
            P.nturn = turns;
            mark(0);
            if (q.sched == kSchedStaged) launch_fused_staged(P, q.variant, C->hot.p, (int)L0->desc.size(), grid, s);
            else launch_fused(P, q.variant, grid, s);
            mark(1);
            launches++;
        } else {
            // one turn: local ranges through the fused kernel, wake elements by their kernels
            int a = q.e0;
            while (a < q.e1) {
                int b = a;
                while (b < q.e1 && !is_collective(L0->desc[b].type)) b++;
                if (b > a) {
                    P.e0 = a;
                    P.e1 = b;
                    P.nturn = 1;
                    mark(0);
                    if (q.sched == kSchedStaged)
                        launch_fused_staged(P, q.variant, C->hot.p, (int)L0->desc.size(), grid, s);
                    else
                        launch_fused(P, q.variant, grid, s);
                    mark(1);
                    launch_fill_i32(cnt + 2, 0, 1, s);  // chunk counter for the next range
                    launches += 2;
                }
                if (b < q.e1) { coll(b); b++; }
                a = b;
            }
        }
        launch_compact(live, cnt + 0, q.st, cnt + 2, cnt + 3, turns, cnt + 5, s);
        launches++;
    } else if (q.mode == ACCEL_MODE_EXACT) {
        if (!has_collective(L0, q.e0, q.e1)) {
            mark(0);
            launch_exact(P, q.e0, q.e1, turns, cnt + 3, true, s);
            mark(1);
            launches += 2;
        } else {
            // one turn: local ranges in one launch each, wake elements by their kernels
            int a = q.e0;
            while (a < q.e1) {
                int b = a;
                while (b < q.e1 && !is_collective(L0->desc[b].type)) b++;
                if (b > a) {
                    mark(0);
                    launch_exact(P, a, b, 1, cnt + 3, false, s);
                    mark(1);
                    launches++;
                }
                if (b < q.e1) { coll(b); b++; }
                a = b;
            }
            launch_plain_turn_end(P, cnt + 3, s);
            launches += 2;
        }
    } else {
        for (int k = q.e0; k < q.e1; k++) {
            if (is_collective(L0->desc[k].type)) {
                coll(k);
            } else {
                mark(0);
                launch_plain_elem(P, k, cnt + 3, s);
                mark(1);
                launches++;
            }
        }
        launch_plain_turn_end(P, cnt + 3, s);
        launches += 2;
    }
    return coll_status;
}

static int capture_part(accel_ctx* C, const CoreReq& q, int part, int turns, cudaGraphExec_t* out,
                        int& launches) {
    cudaStream_t s = C->stream;
    cudaGraph_t graph = nullptr;
    cudaError_t ce = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) return fail(ACCEL_E_CUDA, std::string("begin capture: ") + cudaGetErrorString(ce));
    int st = emit_part(C, q, part, turns, s, [](int) {}, launches);
    ce = cudaStreamEndCapture(s, &graph);
    if (st) { if (graph) cudaGraphDestroy(graph); return st; }
    if (ce != cudaSuccess) return fail(ACCEL_E_CUDA, std::string("end capture: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return fail(ACCEL_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    return ACCEL_OK;
}

static int run_core_plan(accel_ctx* C, const CoreReq& q, cudaStream_t user);

static int run_core(accel_ctx* C, const CoreReq& q, cudaStream_t user) {
    int s;
    if ((s = C->live0.ensure(sizeof(int32_t) * std::max<int64_t>(1, q.ntot)))) return s;
    const bool fresh_cnt = C->cnt.p == nullptr;
    if ((s = C->cnt.ensure(sizeof(int32_t) * 16))) return s;
    if (fresh_cnt) CK(cudaMemsetAsync(C->cnt.p, 0, sizeof(int32_t) * 16, C->stream));  // [6]: a count kept
    if ((s = C->scratch.ensure(sizeof(double) * kScratchDoubles))) return s;
    bool tw = false;
    for (int k = q.e0; k < q.e1; k++) tw |= q.lines[0]->desc[k].type == ACCEL_TRANSWAKE;
    if (tw && C->comm && C->nranks > 1 && q.mode != ACCEL_MODE_FUSED)
        return fail(ACCEL_E_UNSUPPORTED, "the pair-sum transverse wake of the plain and exact modes acts within "
                                         "one rank; a bunch spread over ranks takes the fused mode");
    if (tw && q.mode == ACCEL_MODE_FUSED) {
        // the transverse wake's entries per rank and the particles of all ranks (exchanged when a
        // communicator is set: every rank takes this step, same lattice), then its sort and scan
        // scratch, sized before any graph is captured
        int64_t slots = q.ntot, all = q.ntot;
        if (C->comm) {
            int64_t* d = (int64_t*)C->scratch.p;
            int64_t h[2] = {q.ntot, q.ntot};
            CK(cudaMemcpyAsync(d, h, sizeof h, cudaMemcpyHostToDevice, C->stream));
            ncclComm_t cm = (ncclComm_t)C->comm;
            ncclResult_t r = nccl().AllReduce(d, d, 1, ncclInt64, ncclMax, cm, C->stream);
            if (r == ncclSuccess) r = nccl().AllReduce(d + 1, d + 1, 1, ncclInt64, ncclSum, cm, C->stream);
            if (r != ncclSuccess) return nccl_fail("ncclAllReduce (transverse wake sizes)", r);
            CK(cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, C->stream));
            CK(cudaStreamSynchronize(C->stream));
            slots = h[0];
            all = h[1];
        }
        const int nr = C->comm ? C->nranks : 1;
        if (std::max<int64_t>(1, slots) * nr > INT32_MAX)
            return fail(ACCEL_E_TOO_LARGE, "transverse wake: more than 2^31 entries over all ranks");
        C->tw_slots = std::max<int64_t>(1, slots);
        C->tw_ntot_all = all;
        if ((s = C->tw_scratch.ensure(tw_sorted_scratch_bytes(C->tw_slots, nr, C->comm != nullptr)))) return s;
    }
    if ((s = C->iscratch.ensure(sizeof(int32_t) * 4096))) return s;
    if (q.variant < 0 || q.variant >= kNumFusedVariants) return fail(ACCEL_E_INVALID, "bad variant");
    CoreReq qs = q;
    if (q.mode == ACCEL_MODE_FUSED && q.sched == kSchedStaged) {
        // the staged schedule: one instance's hot lines per block in shared memory; a line too
        // long for shared memory runs the first schedule instead
        const int ne = (int)q.lines[0]->desc.size();
        const int v = q.variant < kNumStagedVariants ? q.variant : 0;
        const int nb = staged_blocks_per_sm(v, ne);
        if (nb <= 0) {
            qs.sched = 0;
        } else {
            qs.variant = v;
            qs.grid_staged = C->sm_count * nb;
            qs.nrec = (int64_t)q.ninst * ne;
            if ((s = C->hot.ensure((size_t)qs.nrec * 128))) return s;
        }
    }
    if (qs.sched != kSchedStaged && C->bps[qs.variant] == 0) {
        C->bps[qs.variant] = fused_blocks_per_sm(qs.variant);
        if (C->bps[qs.variant] <= 0) return fail(ACCEL_E_CUDA, "fused kernel cannot be resident");
    }
    if (q.mode != ACCEL_MODE_FUSED || qs.sched != kSchedStaged) return run_core_plan(C, qs, user);
    // the staged kernel's bulk copies are waited on with a bounded wait; a wait that ran out sets
    // the error word (cnt[4]) and its block leaves, so the run is checked before returning
    int32_t* err = (int32_t*)C->cnt.p + 4;
    CK(cudaMemsetAsync(err, 0, sizeof(int32_t), C->stream));
    if ((s = run_core_plan(C, qs, user))) return s;
    int32_t h = 0;
    CK(cudaMemcpyAsync(&h, err, sizeof h, cudaMemcpyDeviceToHost, C->stream));
    CK(cudaStreamSynchronize(C->stream));
    if (h) return fail(ACCEL_E_TIMEOUT, "a shared-memory staging copy did not complete in its bounded wait");
    return ACCEL_OK;
}

// Issue a prepared request (buffers sized, schedule resolved): as graphs, or directly with events.
static int run_core_plan(accel_ctx* C, const CoreReq& q, cudaStream_t user) {
    const Plan plan = make_plan(q, has_collective(q.lines[0], q.e0, q.e1));
    // order after the caller's prior work on `user`, run on the private stream, then order the
    // caller's stream after ours (user may be 0, the legacy default stream)
    if (user != C->stream) {
        CK(cudaEventRecord(C->ev0, user));
        CK(cudaStreamWaitEvent(C->stream, C->ev0, 0));
    }
    if (C->profile) {
        for (cudaEvent_t e : C->prof_events) cudaEventDestroy(e);
        C->prof_events.clear();
        int launches = 0;
        auto mark = [&](int) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            cudaEventRecord(e, C->stream);
            C->prof_events.push_back(e);
        };
        cudaEvent_t w0, w1;
        cudaEventCreate(&w0);
        cudaEventCreate(&w1);
        cudaEventRecord(w0, C->stream);
        int st = emit_part(C, q, PART_PRE, 0, C->stream, mark, launches);
        for (int i = 0; i < plan.nbody && !st; i++) st = emit_part(C, q, PART_BODY, plan.seg, C->stream, mark, launches);
        if (!st && plan.tail) st = emit_part(C, q, PART_TAIL, plan.tail, C->stream, mark, launches);
        if (!st) st = emit_part(C, q, PART_POST, 0, C->stream, mark, launches);
        cudaEventRecord(w1, C->stream);
        C->prof_events.push_back(w0);
        C->prof_events.push_back(w1);
        C->launches += launches;
        if (st) return st;
    } else {
        GraphKey key;
        key.v = {(int64_t)q.mode, (int64_t)q.ninst, q.ntot, (int64_t)q.e0, (int64_t)q.e1, (int64_t)q.nturn,
                 (int64_t)q.variant, (int64_t)plan.seg, (int64_t)q.sched, (int64_t)(intptr_t)q.st, (int64_t)(intptr_t)q.loss,
                 (int64_t)(intptr_t)q.tables, (int64_t)(intptr_t)q.tbl_off, (int64_t)(intptr_t)q.pinst,
                 (int64_t)q.probe, (int64_t)(intptr_t)C->live0.p, (int64_t)(intptr_t)C->cnt.p,
                 (int64_t)(intptr_t)C->scratch.p, (int64_t)(intptr_t)C->iscratch.p,
                 (int64_t)(intptr_t)C->tw_scratch.p, (int64_t)C->tw_scratch.bytes, C->tw_slots, C->tw_ntot_all,
                 (int64_t)(intptr_t)C->comm, (int64_t)(intptr_t)C->hot.p, (int64_t)q.grid_staged};
        for (int i = 0; i < q.ninst && i < 4; i++) {
            key.v.push_back((int64_t)(intptr_t)q.lines[i]);
            key.v.push_back(q.lines[i]->version);
        }
        key.v.push_back((int64_t)q.lines[0]->seed);
        auto it = C->graphs.find(key);
        GraphEntry* g;
        if (it == C->graphs.end()) {
            if (C->graphs.size() > 32) C->graphs.clear();
            auto ins = C->graphs.emplace(key, std::make_unique<GraphEntry>());
            g = ins.first->second.get();
            int st = 0;
            for (int part = PART_PRE; part <= PART_POST && !st; part++) {
                int turns = part == PART_BODY ? plan.seg : part == PART_TAIL ? plan.tail : 0;
                if (part == PART_TAIL && plan.tail == 0) continue;
                if (part == PART_BODY && plan.nbody == 0) continue;
                st = capture_part(C, q, part, turns, &g->exec[part], g->part_launches[part]);
            }
            if (st) { C->graphs.erase(key); return st; }
        } else {
            g = it->second.get();
        }
        CK(cudaGraphLaunch(g->exec[PART_PRE], C->stream));
        for (int i = 0; i < plan.nbody; i++) CK(cudaGraphLaunch(g->exec[PART_BODY], C->stream));
        if (plan.tail) CK(cudaGraphLaunch(g->exec[PART_TAIL], C->stream));
        CK(cudaGraphLaunch(g->exec[PART_POST], C->stream));
        C->launches += g->part_launches[PART_PRE] + (int64_t)plan.nbody * g->part_launches[PART_BODY] +
                       (plan.tail ? g->part_launches[PART_TAIL] : 0) + g->part_launches[PART_POST];
    }
    if (user != C->stream) {
        CK(cudaEventRecord(C->ev1, C->stream));
        CK(cudaStreamWaitEvent(user, C->ev1, 0));
    }
    return ACCEL_OK;
}

// Untuned jobs run variant 4 (128 threads, 5 blocks per SM; the autotuner's choice on the batched
// DA benchmark and the fastest on a 2^20-particle bunch with a per-turn wake) with 8-turn segments.
constexpr int kDefaultVariant = 4, kDefaultSeg = 8;

static void default_tile(accel_ctx* C, int& variant, int& seg, int& sched) {
    variant = C->tile_variant >= 0 ? C->tile_variant : kDefaultVariant;
    seg = C->tile_seg > 0 ? C->tile_seg : kDefaultSeg;
    sched = C->tile_sched >= 0 ? C->tile_sched : 0;
}

// ------------------------------------------------------------------------------------------
// C-ABI
// ------------------------------------------------------------------------------------------
extern "C" {

const char* accel_status_string(int s) {
    switch (s) {
    case ACCEL_OK: return "ok";
    case ACCEL_E_INVALID: return "invalid argument";
    case ACCEL_E_UNSUPPORTED: return "unsupported element or mode";
    case ACCEL_E_CUDA: return "CUDA runtime error";
    case ACCEL_E_NOMEM: return "out of memory";
    case ACCEL_E_IO: return "lattice I/O error";
    case ACCEL_E_TIMEOUT: return "bounded device wait ran out";
    case ACCEL_E_NODEVICE: return "no CUDA device";
    case ACCEL_E_TOO_LARGE: return "request exceeds a fixed capacity";
    default: return "unknown status";
    }
}

const char* accel_last_error(void) { return g_last_error.c_str(); }

int accel_version(void) { return 10000; }

int accel_device_count(int* n) {
    if (!n) return fail(ACCEL_E_INVALID, "n is NULL");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) { cudaGetLastError(); c = 0; }
    *n = c;
    return ACCEL_OK;
}

int accel_ctx_create(int device, accel_ctx** out) {
    if (!out) return fail(ACCEL_E_INVALID, "out is NULL");
    *out = nullptr;
    int n = 0;
    accel_device_count(&n);
    if (n <= 0) return fail(ACCEL_E_NODEVICE, "no CUDA device is visible");
    if (device < 0 || device >= n) return fail(ACCEL_E_INVALID, "device index out of range");
    std::unique_ptr<accel_ctx> C(new accel_ctx());
    C->device = device;
    CK(cudaSetDevice(device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    C->sm_count = prop.multiProcessorCount;
    if (prop.major < 10) return fail(ACCEL_E_UNSUPPORTED, "this build targets sm_100a (B200)");
    CK(cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&C->ev0, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&C->ev1, cudaEventDisableTiming));
    *out = C.release();
    return ACCEL_OK;
}

}  // extern "C"

namespace accel {
void ctx_unref(accel_ctx* C) {
    if (C->refs.fetch_sub(1) != 1) return;
    cudaSetDevice(C->device);
    cudaStreamSynchronize(C->stream);
    if (C->comm) nccl().CommDestroy((ncclComm_t)C->comm);
    delete C;
}

void line_unref(accel_line* L) {
    if (L->refs.fetch_sub(1) != 1) return;
    accel_ctx* C = L->ctx;
    {
        std::lock_guard<std::mutex> lk(C->mu);
        cudaSetDevice(C->device);
        cudaStreamSynchronize(C->stream);
        C->graphs.clear();
        L->d_tbl.release();
        L->d_aux.release();
        L->d_rng.release();
        delete L;
    }
    ctx_unref(C);
}
}  // namespace accel

extern "C" {

int accel_ctx_destroy(accel_ctx* C) {
    if (!C) return ACCEL_OK;
    accel::ctx_unref(C);
    return ACCEL_OK;
}

int accel_nccl_unique_id(unsigned char* id) {
    if (!id) return fail(ACCEL_E_INVALID, "id is NULL");
    NcclApi& api = nccl();
    if (!api.ok) return fail(ACCEL_E_UNSUPPORTED, api.err);
    ncclUniqueId u;
    ncclResult_t r = api.GetUniqueId(&u);
    if (r != ncclSuccess) return nccl_fail("ncclGetUniqueId", r);
    std::memcpy(id, u.internal, NCCL_UNIQUE_ID_BYTES);
    return ACCEL_OK;
}

int accel_ctx_set_comm(accel_ctx* C, const unsigned char* id, int nranks, int rank) {
    if (!C || !id || nranks < 1 || rank < 0 || rank >= nranks) return fail(ACCEL_E_INVALID, "bad argument");
    NcclApi& api = nccl();
    if (!api.ok) return fail(ACCEL_E_UNSUPPORTED, api.err);
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    CK(cudaStreamSynchronize(C->stream));
    if (C->comm) {
        api.CommDestroy((ncclComm_t)C->comm);
        C->comm = nullptr;
        C->nranks = 1;
        C->rank = 0;
    }
    C->graphs.clear();
    ncclUniqueId u;
    std::memcpy(u.internal, id, NCCL_UNIQUE_ID_BYTES);
    ncclComm_t cm = nullptr;
    ncclResult_t r = api.CommInitRank(&cm, nranks, u, rank);
    if (r != ncclSuccess) return nccl_fail("ncclCommInitRank", r);
    C->comm = cm;
    C->nranks = nranks;
    C->rank = rank;
    return ACCEL_OK;
}

// ---- lattice files -----------------------------------------------------------------------
static int export_desc(const std::vector<accel_elem_desc>& v, accel_elem_desc** elems, int* n) {
    *elems = (accel_elem_desc*)std::malloc(std::max<size_t>(1, v.size()) * sizeof(accel_elem_desc));
    if (!*elems) return fail(ACCEL_E_NOMEM, "malloc");
    if (!v.empty()) std::memcpy(*elems, v.data(), v.size() * sizeof(accel_elem_desc));
    *n = (int)v.size();
    return ACCEL_OK;
}

int accel_lattice_parse(const char* text, accel_elem_desc** elems, int* n) {
    if (!text || !elems || !n) return fail(ACCEL_E_INVALID, "NULL argument");
    std::vector<accel_elem_desc> v;
    std::string err;
    int s = parse_lattice(text, v, err);
    if (s) return fail(s, err);
    return export_desc(v, elems, n);
}

int accel_lattice_read(const char* path, accel_elem_desc** elems, int* n) {
    if (!path || !elems || !n) return fail(ACCEL_E_INVALID, "NULL argument");
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) return fail(ACCEL_E_IO, std::string("Exception opening/reading file:") + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return accel_lattice_parse(ss.str().c_str(), elems, n);
}

int accel_lattice_write(const char* path, const accel_elem_desc* elems, int n, int precision) {
    if (!path || (!elems && n > 0) || n < 0) return fail(ACCEL_E_INVALID, "bad argument");
    if (precision <= 0) precision = 17;
    std::ofstream f(path, std::ios::binary);
    if (!f.good()) return fail(ACCEL_E_IO, std::string("cannot write ") + path);
    f << format_lattice(elems, n, precision);
    return f.good() ? ACCEL_OK : fail(ACCEL_E_IO, "write failed");
}

void accel_lattice_free(accel_elem_desc* elems) { std::free(elems); }

int accel_elem_default(int type, accel_elem_desc* out) {
    if (!out || type < ACCEL_DRIFT || type > ACCEL_LONGWAKE) return fail(ACCEL_E_INVALID, "bad type");
    default_desc(type, out);
    return ACCEL_OK;
}

// ---- lines -------------------------------------------------------------------------------
int accel_line_create(accel_ctx* C, const accel_elem_desc* elems, int n, accel_line** out) {
    if (!C || !out || n < 0 || (n > 0 && !elems)) return fail(ACCEL_E_INVALID, "bad argument");
    std::unique_ptr<accel_line> L(new accel_line());
    L->ctx = C;
    L->desc.assign(elems, elems + n);
    L->dirty = true;
    std::lock_guard<std::mutex> lk(C->mu);
    int s = line_sync(L.get());
    if (s) return s;
    C->refs.fetch_add(1);
    *out = L.release();
    return ACCEL_OK;
}

int accel_line_destroy(accel_line* L) {
    if (!L) return ACCEL_OK;
    accel::line_unref(L);
    return ACCEL_OK;
}

int accel_line_count(const accel_line* L, int* n) {
    if (!L || !n) return fail(ACCEL_E_INVALID, "NULL argument");
    *n = (int)L->desc.size();
    return ACCEL_OK;
}

int accel_line_get_desc(const accel_line* L, int idx, accel_elem_desc* out) {
    if (!L || !out || idx < 0 || idx >= (int)L->desc.size()) return fail(ACCEL_E_INVALID, "bad index");
    *out = L->desc[(size_t)idx];
    return ACCEL_OK;
}

int accel_line_set_field(accel_line* L, int idx, int field, int index, const double* v) {
    if (!L || !v || idx < 0 || idx >= (int)L->desc.size()) return fail(ACCEL_E_INVALID, "bad index");
    accel_elem_desc& d = L->desc[(size_t)idx];
    int s = desc_set_field(d, field, index, v);
    if (s) return s;
    L->dirty = true;
    return ACCEL_OK;
}

int accel_line_get_field(const accel_line* L, int idx, int field, int index, double* v) {
    if (!L || !v || idx < 0 || idx >= (int)L->desc.size()) return fail(ACCEL_E_INVALID, "bad index");
    return desc_get_field(L->desc[(size_t)idx], field, index, v);
}

int accel_line_set_flags(accel_line* L, int rad_flag, int cavity_on, int wake_on) {
    if (!L) return fail(ACCEL_E_INVALID, "NULL line");
    apply_flags(L->desc.data(), (int)L->desc.size(), rad_flag, cavity_on, wake_on);
    L->dirty = true;
    return ACCEL_OK;
}

int accel_line_set_crab_onoff(accel_line* L, int on, int* count) {
    if (!L) return fail(ACCEL_E_INVALID, "NULL line");
    int n = 0;
    for (auto& d : L->desc)  // ALine::set_crab_onoff, aline.cpp:441-450
        if (d.type == ACCEL_CRABCAV) { d.flags = on ? 1 : 0; n++; }
    if (count) *count = n;
    L->dirty = true;
    return ACCEL_OK;
}

int accel_line_set_energy(accel_line* L, double en) {
    if (!L) return fail(ACCEL_E_INVALID, "NULL line");
    for (auto& d : L->desc) {  // ALine::setenergy, aline.cpp:220-257
        if (d.type == ACCEL_CAVITY) d.f[3] = en;
        else if (d.type == ACCEL_CRABCAV) d.f[4] = en;
        else if (d.type == ACCEL_RFMULT) d.f[2] = en;
        else if (d.type == ACCEL_IDEALWIG) d.f[3] = en;
        else if (d.type == ACCEL_BENDMPOLE) d.f[3] = en;
        else if (d.type == ACCEL_TRANSWAKE) d.f[0] = en;
        else if (d.type == ACCEL_LONGWAKE) d.f[0] = en;
    }
    L->dirty = true;
    return ACCEL_OK;
}

int accel_line_set_seed(accel_line* L, uint64_t seed) {
    if (!L) return fail(ACCEL_E_INVALID, "NULL line");
    L->seed = seed;
    std::lock_guard<std::mutex> lk(L->ctx->mu);
    cudaSetDevice(L->ctx->device);
    int s = line_sync(L);
    if (s) return s;
    CK(cudaMemset(L->d_rng.p, 0, sizeof(int32_t) * 2));
    return ACCEL_OK;
}

// ---- tracking ----------------------------------------------------------------------------
int accel_track(accel_line* L, double* r, int layout, int N, int st, int ed, int nturn,
                int32_t* loss_turn, int mode, void* stream) {
    if (!L || (!r && N > 0) || N < 0 || nturn < 0) return fail(ACCEL_E_INVALID, "bad argument");
    if (layout != ACCEL_LAYOUT_AOS && layout != ACCEL_LAYOUT_SOA) return fail(ACCEL_E_INVALID, "bad layout");
    if (mode != ACCEL_MODE_FUSED && mode != ACCEL_MODE_PLAIN && mode != ACCEL_MODE_EXACT)
        return fail(ACCEL_E_INVALID, "bad mode");
    const int ne = (int)L->desc.size();
    if (st < 0 || ed > ne || st > ed) return fail(ACCEL_E_INVALID, "element range out of bounds");
    accel_ctx* C = L->ctx;
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    int s = line_sync(L);
    if (s) return s;
    if ((s = check_supported(L, st, ed))) return s;
    if (N == 0 || nturn == 0 || st == ed) {
        // nothing runs: no particle is recorded as lost by this call
        if (loss_turn && N > 0) {
            if (is_device_ptr(loss_turn)) {
                launch_fill_i32(loss_turn, -1, N, C->stream);
                CK(cudaStreamSynchronize(C->stream));
            } else {
                for (int i = 0; i < N; i++) loss_turn[i] = -1;
            }
        }
        return ACCEL_OK;
    }
    cudaStream_t user = (cudaStream_t)stream;  // NULL: the legacy default stream
    const bool rdev = is_device_ptr(r);
    const bool ldev = loss_turn ? is_device_ptr(loss_turn) : false;
    const size_t nb = sizeof(double) * 6 * (size_t)N;
    if ((s = C->state.ensure(nb))) return s;
    if ((s = C->loss.ensure(sizeof(int32_t) * (size_t)N))) return s;
    double* soa = (double*)C->state.p;
    double* dev_in = nullptr;
    if (rdev) {
        if (layout == ACCEL_LAYOUT_SOA) soa = r;
        else dev_in = r;
    } else {
        if ((s = C->aos.ensure(nb))) return s;
        CK(cudaMemcpyAsync(C->aos.p, r, nb, cudaMemcpyHostToDevice, user));
        if (layout == ACCEL_LAYOUT_SOA) {
            CK(cudaMemcpyAsync(soa, C->aos.p, nb, cudaMemcpyDeviceToDevice, user));
        } else {
            dev_in = (double*)C->aos.p;
        }
    }
    if (dev_in) launch_aos_to_soa(dev_in, soa, N, user);
    int32_t* dloss = ldev ? loss_turn : (int32_t*)C->loss.p;
    CoreReq q{};
    accel_line* lines[1] = {L};
    q.lines = lines;
    q.ninst = 1;
    q.tables = (const DevElem*)L->d_tbl.p;
    q.st = soa;
    q.ntot = N;
    q.loss = dloss;
    q.e0 = st;
    q.e1 = ed;
    q.nturn = nturn;
    q.mode = mode;
    default_tile(C, q.variant, q.seg, q.sched);
    auto tk = C->tuned.find(tune_key(lines, 1, N, nturn));
    if (tk != C->tuned.end() && C->tile_variant < 0) {
        q.variant = tk->second[0]; q.seg = tk->second[1]; q.sched = tk->second[2];
    }
    if ((s = run_core(C, q, user))) return s;
    if (dev_in) launch_soa_to_aos(soa, dev_in, N, user);
    if (!rdev) {
        if (layout == ACCEL_LAYOUT_SOA) CK(cudaMemcpyAsync(r, soa, nb, cudaMemcpyDeviceToHost, user));
        else CK(cudaMemcpyAsync(r, C->aos.p, nb, cudaMemcpyDeviceToHost, user));
    }
    if (loss_turn && !ldev)
        CK(cudaMemcpyAsync(loss_turn, dloss, sizeof(int32_t) * (size_t)N, cudaMemcpyDeviceToHost, user));
    if (!rdev || (loss_turn && !ldev)) CK(cudaStreamSynchronize(user));
    CK(cudaGetLastError());
    return ACCEL_OK;
}

static int stage_batch(accel_ctx* C, accel_line* const* lines, int ninst, const int64_t* part_off,
                       int64_t ntot, const DevElem** tables, const int32_t** tbl_off,
                       const int32_t** pinst, cudaStream_t s) {
    const int ne = (int)lines[0]->desc.size();
    // concatenated tables: reuse when the same lines at the same versions are staged again
    BatchKey bk;
    bk.v.push_back(ntot);
    for (int i = 0; i < ninst; i++) {
        bk.v.push_back((int64_t)(intptr_t)lines[i]);
        bk.v.push_back(lines[i]->version);
        bk.v.push_back(part_off[i]);
    }
    bk.v.push_back(part_off[ninst]);
    int st;
    if (!(C->batch_key == bk)) {
        if ((st = C->tables.ensure(sizeof(DevElem) * (size_t)ne * ninst))) return st;
        if ((st = C->tbl_off.ensure(sizeof(int32_t) * (size_t)ninst))) return st;
        if ((st = C->pinst.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(1, ntot)))) return st;
        std::vector<int32_t> off((size_t)ninst);
        std::vector<int32_t> pi((size_t)ntot);
        for (int i = 0; i < ninst; i++) {
            CK(cudaMemcpyAsync((DevElem*)C->tables.p + (size_t)i * ne, lines[i]->d_tbl.p,
                               sizeof(DevElem) * ne, cudaMemcpyDeviceToDevice, s));
            off[(size_t)i] = i * ne;
            for (int64_t p = part_off[i]; p < part_off[i + 1]; p++) pi[(size_t)p] = i;
        }
        CK(cudaMemcpyAsync(C->tbl_off.p, off.data(), sizeof(int32_t) * ninst, cudaMemcpyHostToDevice, s));
        if (ntot > 0)
            CK(cudaMemcpyAsync(C->pinst.p, pi.data(), sizeof(int32_t) * ntot, cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
        C->batch_key = bk;
    }
    *tables = (const DevElem*)C->tables.p;
    *tbl_off = (const int32_t*)C->tbl_off.p;
    *pinst = (const int32_t*)C->pinst.p;
    return ACCEL_OK;
}

static int check_batch(accel_line* const* lines, int ninst, const int64_t* part_off, int64_t ntot) {
    if (!lines || ninst <= 0 || !part_off) return fail(ACCEL_E_INVALID, "bad batch");
    accel_ctx* C = lines[0]->ctx;
    const size_t ne = lines[0]->desc.size();
    if (part_off[0] != 0 || part_off[ninst] != ntot) return fail(ACCEL_E_INVALID, "part_off must run 0..ntot");
    for (int i = 0; i < ninst; i++) {
        if (!lines[i] || lines[i]->ctx != C) return fail(ACCEL_E_INVALID, "lines from different contexts");
        if (lines[i]->desc.size() != ne) return fail(ACCEL_E_INVALID, "lines differ in element count");
        if (part_off[i + 1] < part_off[i]) return fail(ACCEL_E_INVALID, "part_off not monotone");
        if (ninst > 1)
            for (auto& d : lines[i]->desc)
                if (is_collective(d.type)) return fail(ACCEL_E_UNSUPPORTED, "wake elements need a single-instance launch");
    }
    if (ntot > INT32_MAX) return fail(ACCEL_E_TOO_LARGE, "more than 2^31 particles");
    return ACCEL_OK;
}

int accel_track_batched(accel_line* const* lines, int ninst, const int64_t* part_off, double* r_soa,
                        int64_t ntot, int nturn, int32_t* loss_turn, int mode, void* stream) {
    int s = check_batch(lines, ninst, part_off, ntot);
    if (s) return s;
    if (!r_soa || nturn < 0) return fail(ACCEL_E_INVALID, "bad argument");
    if (mode != ACCEL_MODE_FUSED && mode != ACCEL_MODE_PLAIN && mode != ACCEL_MODE_EXACT)
        return fail(ACCEL_E_INVALID, "bad mode");
    accel_ctx* C = lines[0]->ctx;
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    for (int i = 0; i < ninst; i++) {
        if ((s = line_sync(lines[i]))) return s;
        if ((s = check_supported(lines[i], 0, (int)lines[i]->desc.size()))) return s;
    }
    // host or device arrays: host ones are staged through the context's buffers, one
    // cudaMemcpyAsync each way per array, and the call returns once they are copied back
    const bool rdev = is_device_ptr(r_soa);
    const bool ldev = loss_turn ? is_device_ptr(loss_turn) : false;
    if (ntot == 0 || nturn == 0) {
        if (loss_turn && ntot > 0) {  // nothing runs: no particle is recorded as lost
            if (ldev) {
                launch_fill_i32(loss_turn, -1, ntot, C->stream);
                CK(cudaStreamSynchronize(C->stream));
            } else {
                for (int64_t i = 0; i < ntot; i++) loss_turn[i] = -1;
            }
        }
        return ACCEL_OK;
    }
    cudaStream_t user = (cudaStream_t)stream;  // NULL: the legacy default stream
    const size_t nb = sizeof(double) * 6 * (size_t)ntot;
    if ((s = C->loss.ensure(sizeof(int32_t) * (size_t)ntot))) return s;
    if (!rdev) {
        if ((s = C->state.ensure(nb))) return s;
        CK(cudaMemcpyAsync(C->state.p, r_soa, nb, cudaMemcpyHostToDevice, user));
    }
    CoreReq q{};
    q.lines = lines;
    q.ninst = ninst;
    if ((s = stage_batch(C, lines, ninst, part_off, ntot, &q.tables, &q.tbl_off, &q.pinst, C->stream))) return s;
    q.st = rdev ? r_soa : (double*)C->state.p;
    q.ntot = ntot;
    q.loss = ldev ? loss_turn : (int32_t*)C->loss.p;
    q.e0 = 0;
    q.e1 = (int)lines[0]->desc.size();
    q.nturn = nturn;
    q.mode = mode;
    default_tile(C, q.variant, q.seg, q.sched);
    auto tk = C->tuned.find(tune_key(lines, ninst, ntot, nturn));
    if (tk != C->tuned.end() && C->tile_variant < 0) {
        q.variant = tk->second[0]; q.seg = tk->second[1]; q.sched = tk->second[2];
    }
    if ((s = run_core(C, q, user))) return s;
    if (!rdev) CK(cudaMemcpyAsync(r_soa, q.st, nb, cudaMemcpyDeviceToHost, user));
    if (loss_turn && !ldev)
        CK(cudaMemcpyAsync(loss_turn, q.loss, sizeof(int32_t) * (size_t)ntot, cudaMemcpyDeviceToHost, user));
    if (!rdev || (loss_turn && !ldev)) CK(cudaStreamSynchronize(user));
    CK(cudaGetLastError());
    return ACCEL_OK;
}

// Autotuner: times the fused kernel variants (block size x register cap) on a short probe, then
// the segment length (compaction cadence) on a longer one, on a scratch copy of the state; the
// winner is cached per (lines, particle count, turn count) and used by later calls.
int accel_autotune(accel_line* const* lines, int ninst, const int64_t* part_off, const double* r_soa,
                   int64_t ntot, int* tile_out3) {
    int s = check_batch(lines, ninst, part_off, ntot);
    if (s) return s;
    if (!r_soa || !is_device_ptr(r_soa)) return fail(ACCEL_E_INVALID, "r_soa must be device memory");
    accel_ctx* C = lines[0]->ctx;
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    for (int i = 0; i < ninst; i++)
        if ((s = line_sync(lines[i]))) return s;
    const size_t nb = sizeof(double) * 6 * (size_t)ntot;
    if ((s = C->probe_state.ensure(nb))) return s;
    if ((s = C->loss.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(1, ntot)))) return s;
    CoreReq q{};
    q.lines = lines;
    q.ninst = ninst;
    if ((s = stage_batch(C, lines, ninst, part_off, ntot, &q.tables, &q.tbl_off, &q.pinst, C->stream))) return s;
    q.st = (double*)C->probe_state.p;
    q.ntot = ntot;
    q.loss = (int32_t*)C->loss.p;
    q.e0 = 0;
    q.e1 = (int)lines[0]->desc.size();
    q.mode = ACCEL_MODE_FUSED;
    q.probe = true;
    auto time_it = [&](int variant, int seg, int sched, int turns, float* ms) -> int {
        q.variant = variant;
        q.seg = seg;
        q.sched = sched;
        q.nturn = turns;
        CK(cudaMemcpyAsync(q.st, r_soa, nb, cudaMemcpyDeviceToDevice, C->stream));
        int st2 = run_core(C, q, C->stream);  // builds the (untimed) graphs on first use
        if (st2) return st2;
        CK(cudaMemcpyAsync(q.st, r_soa, nb, cudaMemcpyDeviceToDevice, C->stream));
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, C->stream);
        st2 = run_core(C, q, C->stream);
        cudaEventRecord(b, C->stream);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return st2;
    };
    // variants: 16-turn probes (long enough for the first losses to thin the live list), each
    // the better of two runs; a later candidate must beat the best so far by 2 % (timing noise
    // of a few tenths of a percent would otherwise pick variants at random between runs)
    int best_v = 0, best_sched = 0;
    float best = 1e30f;
    for (int sched = 0; sched < kNumSched; sched++)
        for (int v = 0; v < (sched == kSchedStaged ? kNumStagedVariants : kNumFusedVariants); v++) {
            float ms = 1e30f;
            for (int rep = 0; rep < 2; rep++) {
                float m1 = 0;
                if ((s = time_it(v, 4, sched, 16, &m1))) return s;
                ms = std::min(ms, m1);
            }
            if (ms < best * 0.98f) { best = ms; best_v = v; best_sched = sched; }
        }
    // turns per segment: 64-turn probes, each the better of two runs, starting from the untuned
    // default of 8 and moving outward; another length must win by 2 % (64 turns from the start
    // over-weight the early turns, where most losses fall and short segments compact sooner)
    int best_seg = 8;
    best = 1e30f;
    for (int seg : {8, 4, 16, 2, 32, 1}) {
        float ms = 1e30f;
        for (int rep = 0; rep < 2; rep++) {
            float m1 = 0;
            if ((s = time_it(best_v, seg, best_sched, 64, &m1))) return s;
            ms = std::min(ms, m1);
        }
        if (ms < best * (seg == 8 ? 1.0f : 0.98f)) { best = ms; best_seg = seg; }
    }
    C->graphs.clear();
    C->tuned[tune_key(lines, ninst, ntot, -1)] = {best_v, best_seg, best_sched};
    if (tile_out3) {
        tile_out3[0] = best_sched == kSchedStaged ? staged_variant_info(best_v).block : fused_variant_info(best_v).block;
        tile_out3[1] = best_seg;
        tile_out3[2] = best_v + 100 * best_sched;
    }
    return ACCEL_OK;
}

int accel_set_tile(accel_ctx* C, int block, int seg_turns, int variant) {
    if (!C) return fail(ACCEL_E_INVALID, "NULL ctx");
    std::lock_guard<std::mutex> lk(C->mu);
    int sched = -1;
    if (variant >= 100) { sched = variant / 100; variant %= 100; }
    if (variant >= kNumFusedVariants || sched >= kNumSched ||
        (sched == kSchedStaged && variant >= kNumStagedVariants))
        return fail(ACCEL_E_INVALID, "variant out of range");
    C->tile_sched = sched;
    if (variant < 0 && block > 0) {
        for (int v = 0; v < kNumFusedVariants; v++)
            if (fused_variant_info(v).block == block) { variant = v; break; }
    }
    C->tile_variant = variant;
    C->tile_seg = seg_turns;
    C->graphs.clear();
    return ACCEL_OK;
}

int accel_set_stage_wait(accel_ctx* C, int probes) {
    if (!C) return fail(ACCEL_E_INVALID, "NULL ctx");
    std::lock_guard<std::mutex> lk(C->mu);
    C->stage_wait = probes;
    C->graphs.clear();  // the limit is a launch parameter of the captured graphs
    return ACCEL_OK;
}

int accel_get_tile(accel_ctx* C, int* t) {
    if (!C || !t) return fail(ACCEL_E_INVALID, "NULL argument");
    int v, s, sc;
    default_tile(C, v, s, sc);
    t[0] = sc == kSchedStaged ? staged_variant_info(v).block : fused_variant_info(v).block;
    t[1] = s;
    t[2] = v + 100 * sc;
    return ACCEL_OK;
}

// ---- transfer matrices ------------------------------------------------------------------------
int accel_m66_at(accel_line* L, int st, int ed, const double* r0, int method, double delta, double* m) {
    if (!L || !r0 || !m) return fail(ACCEL_E_INVALID, "NULL argument");
    if (method != 0 && method != 1) return fail(ACCEL_E_INVALID, "method must be 0 or 1");
    const int ne = (int)L->desc.size();
    if (st < 0 || ed > ne || st > ed) return fail(ACCEL_E_INVALID, "element range out of bounds");
    accel_ctx* C = L->ctx;
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    int s = line_sync(L);
    if (s) return s;
    if ((s = check_supported(L, st, ed))) return s;
    for (int k = st; k < ed; k++)
        if (is_collective(L->desc[k].type) && L->desc[k].flags)
            return fail(ACCEL_E_UNSUPPORTED, "a transfer matrix through an active wake is not defined");
    if ((s = C->scratch.ensure(sizeof(double) * kScratchDoubles))) return s;
    double* d = (double*)C->scratch.p;
    CK(cudaMemcpyAsync(d, r0, 6 * sizeof(double), cudaMemcpyHostToDevice, C->stream));
    launch_m66((const DevElem*)L->d_tbl.p, st, ed, d, delta, method, d + 8, C->stream);
    C->launches += 1;
    CK(cudaMemcpyAsync(m, d + 8, 36 * sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    CK(cudaStreamSynchronize(C->stream));
    CK(cudaGetLastError());
    return ACCEL_OK;
}

int accel_m66(accel_line* L, int st, int ed, double dpp, double delta, int method, double* m) {
    double r0[6] = {0, 0, 0, 0, 0, dpp};
    return accel_m66_at(L, st, ed, r0, method, delta, m);
}

int accel_m66_knob(accel_line* L, int st, int ed, const double* r0, int nk, const int32_t* elem,
                   const int32_t* field, const int32_t* index, double* m, double* dm) {
    if (!L || !r0 || !m || !dm || nk <= 0 || !elem || !field || !index) return fail(ACCEL_E_INVALID, "bad argument");
    const int ne = (int)L->desc.size();
    if (st < 0 || ed > ne || st > ed) return fail(ACCEL_E_INVALID, "element range out of bounds");
    // per-element knob codes: kind * 16 + coefficient index (kind 1 PolynomB, 2 PolynomA, 3 Quad K)
    std::vector<int32_t> code((size_t)ne, 0);
    for (int j = 0; j < nk; j++) {
        const int e = elem[j];
        if (e < 0 || e >= ne) return fail(ACCEL_E_INVALID, "knob element out of range");
        const accel_elem_desc& d = L->desc[(size_t)e];
        int c = 0;
        if (d.type == ACCEL_STRMPOLE && (field[j] == ACCEL_F_POLYNOMB || field[j] == ACCEL_F_POLYNOMA)) {
            if (index[j] < 0 || index[j] >= ACCEL_MAX_MPOLE) return fail(ACCEL_E_INVALID, "multipole index outside 0..9");
            c = (field[j] == ACCEL_F_POLYNOMB ? 1 : 2) * 16 + index[j];
        } else if (d.type == ACCEL_STRMPOLE && field[j] == ACCEL_F_K) {
            c = 1 * 16 + 1;
        } else if (d.type == ACCEL_QUAD && field[j] == ACCEL_F_K) {
            c = 3 * 16;
        } else {
            return fail(ACCEL_E_UNSUPPORTED, std::string("no knob derivative for this field of ") + d.famname);
        }
        if (code[(size_t)e] != 0 && code[(size_t)e] != c)
            return fail(ACCEL_E_UNSUPPORTED, "one knob moves two coefficients of one element");
        code[(size_t)e] = c;
    }
    accel_ctx* C = L->ctx;
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    int s = line_sync(L);
    if (s) return s;
    if ((s = check_supported(L, st, ed))) return s;
    for (int k = st; k < ed; k++)
        if (is_collective(L->desc[k].type) && L->desc[k].flags)
            return fail(ACCEL_E_UNSUPPORTED, "a transfer matrix through an active wake is not defined");
    // scratch: r0 at 0, m at 8, dm at 48, the knob codes from double 128 on
    if ((size_t)ne > (kScratchDoubles - 128) * 2) return fail(ACCEL_E_TOO_LARGE, "too many elements for a knob derivative");
    if ((s = C->scratch.ensure(sizeof(double) * kScratchDoubles))) return s;
    double* d = (double*)C->scratch.p;
    int32_t* dk = (int32_t*)(d + 128);
    CK(cudaMemcpyAsync(d, r0, 6 * sizeof(double), cudaMemcpyHostToDevice, C->stream));
    CK(cudaMemcpyAsync(dk, code.data(), sizeof(int32_t) * code.size(), cudaMemcpyHostToDevice, C->stream));
    launch_m66_knob((const DevElem*)L->d_tbl.p, st, ed, d, dk, d + 8, d + 48, C->stream);
    C->launches += 1;
    CK(cudaMemcpyAsync(m, d + 8, 36 * sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    CK(cudaMemcpyAsync(dm, d + 48, 36 * sizeof(double), cudaMemcpyDeviceToHost, C->stream));
    CK(cudaStreamSynchronize(C->stream));
    CK(cudaGetLastError());
    return ACCEL_OK;
}

// ALine::setrfphase() (aline.cpp:465-501): cavities off, radiation on, one turn of a zero
// particle, phi_s = asin(U0/V_tot), radiation off.  Cavities are left off, as the reference does.
int accel_line_setrfphase(accel_line* L, double* phis_out) {
    if (!L) return fail(ACCEL_E_INVALID, "NULL line");
    apply_flags(L->desc.data(), (int)L->desc.size(), ACCEL_RAD_RAD, 0, -1);
    L->dirty = true;
    double r[6] = {0, 0, 0, 0, 0, 0};
    int s = accel_track(L, r, ACCEL_LAYOUT_AOS, 1, 0, (int)L->desc.size(), 1, nullptr, ACCEL_MODE_PLAIN, nullptr);
    if (s) return s;
    double delta = -r[5];
    apply_flags(L->desc.data(), (int)L->desc.size(), ACCEL_RAD_OFF, -1, -1);
    L->dirty = true;
    double tot_volt = 0, energy = 0;
    int nrf = 0;
    for (auto& d : L->desc)
        if (d.type == ACCEL_CAVITY) { tot_volt += d.f[0]; energy = d.f[3]; nrf++; }
    if (!nrf) return fail(ACCEL_E_INVALID, "cavity not found");
    double phis = std::asin(delta * energy / tot_volt);
    for (auto& d : L->desc)
        if (d.type == ACCEL_CAVITY) d.f[2] = phis;
    if (phis_out) *phis_out = phis;
    return ACCEL_OK;
}

// ---- beam statistics, peak probe, counters ---------------------------------------------------
// sums `count` device doubles over the context's ranks (accel_beam_stat's exchange)
static int stat_allreduce(void* ctx, double* buf, int count, cudaStream_t s) {
    accel_ctx* C = (accel_ctx*)ctx;
    const ncclResult_t r = nccl().AllReduce(buf, buf, (size_t)count, ncclFloat64, ncclSum, (ncclComm_t)C->comm, s);
    return r == ncclSuccess ? 0 : nccl_fail("ncclAllReduce (beam moments)", r);
}

int accel_beam_stat(accel_ctx* C, const double* r, int layout, int N, double* mean, double* sigma,
                    double* cross, int* nlive) {
    if (!C || !r || N <= 0) return fail(ACCEL_E_INVALID, "bad argument");
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    const size_t nb = sizeof(double) * 6 * (size_t)N;
    int s;
    if ((s = C->state.ensure(nb))) return s;
    const bool rdev = is_device_ptr(r);
    const double* soa = r;
    if (!rdev || layout == ACCEL_LAYOUT_AOS) {
        if ((s = C->aos.ensure(nb))) return s;
        if (!rdev) CK(cudaMemcpyAsync(C->aos.p, r, nb, cudaMemcpyHostToDevice, C->stream));
        const double* src = rdev ? r : (const double*)C->aos.p;
        if (layout == ACCEL_LAYOUT_AOS) launch_aos_to_soa(src, (double*)C->state.p, N, C->stream);
        else CK(cudaMemcpyAsync(C->state.p, src, nb, cudaMemcpyDeviceToDevice, C->stream));
        soa = (const double*)C->state.p;
    }
    int nblk = beam_stat_blocks(N);  // <= 1024, so 12 * nblk + 64 fits the fixed scratch
    if ((s = C->scratch.ensure(sizeof(double) * kScratchDoubles))) return s;
    double* part = (double*)C->scratch.p;
    double* out = part + 12 * (size_t)nblk + 32;
    // a context with a communicator holds its rank's part of a bunch: the moments are the
    // bunch's, the two passes' sums added over the ranks (every rank takes this call)
    if ((s = launch_beam_stat(soa, N, part, nblk, out, C->stream, C->comm ? stat_allreduce : nullptr, C)))
        return s;
    C->launches += 5;
    double h[19];
    CK(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, C->stream));
    CK(cudaStreamSynchronize(C->stream));
    for (int k = 0; k < 6; k++) {
        if (mean) mean[k] = h[k];
        if (sigma) sigma[k] = h[6 + k];
        if (cross) cross[k] = h[12 + k];
    }
    if (nlive) *nlive = (int)h[18];
    return ACCEL_OK;
}

int accel_fp64_peak_clocked(accel_ctx* C, double* tflops, double* sm_mhz) {
    if (!C || !tflops) return fail(ACCEL_E_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    float ms = 0;
    double mhz = 0;
    *tflops = fp64_peak_run(C->sm_count, C->stream, &ms, &mhz);
    if (sm_mhz) *sm_mhz = mhz;
    C->launches += 4;  // the warm-up and three timed probes
    CK(cudaGetLastError());
    return ACCEL_OK;
}

int accel_fp64_peak(accel_ctx* C, double* tflops) { return accel_fp64_peak_clocked(C, tflops, nullptr); }

int accel_profile_enable(accel_ctx* C, int on) {
    if (!C) return fail(ACCEL_E_INVALID, "NULL ctx");
    std::lock_guard<std::mutex> lk(C->mu);
    C->profile = on != 0;
    return ACCEL_OK;
}

int accel_profile_read(accel_ctx* C, double* fused_ms, int64_t* n, double* total_ms) {
    if (!C) return fail(ACCEL_E_INVALID, "NULL ctx");
    std::lock_guard<std::mutex> lk(C->mu);
    CK(cudaSetDevice(C->device));
    CK(cudaStreamSynchronize(C->stream));
    double f = 0, tot = 0;
    int64_t cnt = 0;
    const auto& ev = C->prof_events;
    if (C->profile && ev.size() >= 2) {
        size_t m = ev.size() - 2;
        for (size_t i = 0; i + 1 < m; i += 2) {
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
            f += ms;
            cnt++;
        }
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev[m], ev[m + 1]));
        tot = ms;
    }
    if (fused_ms) *fused_ms = f;
    if (n) *n = cnt;
    if (total_ms) *total_ms = tot;
    return ACCEL_OK;
}

int accel_transwake_pair_passes(accel_ctx* C, int64_t* count) {
    if (!C || !count) return fail(ACCEL_E_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(C->mu);
    *count = 0;
    if (!C->cnt.p) return ACCEL_OK;
    CK(cudaSetDevice(C->device));
    int32_t v = 0;
    CK(cudaMemcpyAsync(&v, (int32_t*)C->cnt.p + 6, sizeof v, cudaMemcpyDeviceToHost, C->stream));
    CK(cudaStreamSynchronize(C->stream));
    *count = v;
    return ACCEL_OK;
}

int accel_launch_count(accel_ctx* C, int64_t* count) {
    if (!C || !count) return fail(ACCEL_E_INVALID, "NULL argument");
    *count = C->launches;
    return ACCEL_OK;
}

}  // extern "C"
