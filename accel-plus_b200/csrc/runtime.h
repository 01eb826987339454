// runtime.h — host-side objects behind the opaque C-ABI handles.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <array>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>
#include "engine.h"
#include "kernels.h"

namespace accel {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t nbytes);  // grow-only; contents are not preserved on growth
    void release();
};

struct GraphKey {
    std::vector<int64_t> v;
    bool operator<(const GraphKey& o) const { return v < o.v; }
    bool operator==(const GraphKey& o) const { return v == o.v; }
};
using BatchKey = GraphKey;

struct GraphEntry {
    cudaGraphExec_t exec[4] = {nullptr, nullptr, nullptr, nullptr};  // pre, body, tail, post
    int part_launches[4] = {0, 0, 0, 0};  // this library's kernels per launch of each part
    ~GraphEntry();
};

int line_sync(struct ::accel_line* L);
int desc_set_field(accel_elem_desc& d, int field, int index, const double* v);
int desc_get_field(const accel_elem_desc& d, int field, int index, double* v);
void apply_flags(accel_elem_desc* d, int n, int rad_flag, int cavity_on, int wake_on);
void launch_rng_advance(int32_t* base, int nturn, cudaStream_t s);

}  // namespace accel

// Handles are reference counted so that they may be destroyed in any order: a context counts
// its live lines, a line its live adjoints, and each is released when its own destroy has been
// called and its last child is gone.
struct accel_ctx {
    std::atomic<int> refs{1};
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::mutex mu;
    accel::DevBuf state, aos, loss, live0, cnt, tables, tbl_off, pinst, scratch, iscratch,
        probe_state, tw_scratch, hot;  // hot: the element records' first lines (staged schedule)
    int tile_variant = -1;  // -1: tuned or default
    int tile_seg = 0;       // 0: tuned or default
    int stage_wait = 0;     // staged schedule's first-wait probes (accel_set_stage_wait)
    int tile_sched = -1;    // -1: tuned or default
    int bps[accel::kNumFusedVariants] = {0};
    std::map<accel::GraphKey, std::unique_ptr<accel::GraphEntry>> graphs;
    std::map<accel::GraphKey, std::array<int, 3>> tuned;  // -> (variant, seg, sched)
    accel::BatchKey batch_key;
    int64_t launches = 0;
    bool profile = false;                  // direct launches with events (accel_profile_enable)
    std::vector<cudaEvent_t> prof_events;  // [begin, end] per tracking launch, then whole call
    void* comm = nullptr;                  // NCCL communicator of a bunch spread over GPUs
    int nranks = 1;
    int rank = 0;
    int64_t tw_slots = 0;                  // transverse wake: entries per rank (max particles)
    int64_t tw_ntot_all = 0;               // and the particles of all ranks, set per run
    ~accel_ctx();
};

struct accel_line {
    std::atomic<int> refs{1};
    accel_ctx* ctx = nullptr;
    std::vector<accel_elem_desc> desc;
    std::vector<accel::DevElem> host_tbl;
    accel::DevBuf d_tbl;
    accel::DevBuf d_aux;  // WigTable kick tables of this line, addressed from their records
    accel::DevBuf d_rng;  // [0]: QE turn base, advanced by every tracking call
    bool dirty = true;
    int64_t version = 0;
    uint64_t seed = 0x5EED5EEDull;
};

namespace accel {
inline GraphKey tune_key(::accel_line* const* lines, int ninst, int64_t ntot, int /*nturn*/) {
    GraphKey k;
    k.v = {(int64_t)(intptr_t)lines[0], lines[0]->version, (int64_t)ninst, ntot};
    return k;
}
}  // namespace accel

namespace accel {
void ctx_unref(accel_ctx* C);   // drop one reference; the last one frees the context
void line_unref(accel_line* L);  // drop one reference; the last one frees the line and unrefs its context
}  // namespace accel
