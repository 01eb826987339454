// state_io.cpp — lossless particle-state checkpoints (accel_state_write / accel_state_read).
//
// The reference saves a distribution only as the 6-significant-digit text of Do_Track's
// "Full export" block and reads it back with "Distribution: Load f, format=accel-export", so a
// resumed run starts from rounded coordinates.  These files hold the doubles themselves, so a run
// split at a checkpoint continues bit for bit.
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include "engine.h"

namespace {
struct StateHeader {
    char magic[8];      // "ACCELST1"
    uint32_t version;   // 1
    uint32_t flags;     // bit 0: loss turns follow the coordinates
    int64_t n;          // particles
    int64_t turn;       // turns tracked when the state was written
};
static_assert(sizeof(StateHeader) == 32, "the state header is 32 bytes");
constexpr char kMagic[8] = {'A', 'C', 'C', 'E', 'L', 'S', 'T', '1'};

bool little_endian() {
    const uint16_t one = 1;
    unsigned char b;
    std::memcpy(&b, &one, 1);
    return b == 1;
}
}  // namespace

using accel::fail;

extern "C" int accel_state_write(const char* path, const double* r, int64_t n, int64_t turn,
                                 const int32_t* loss_turn) {
    if (!path || (!r && n > 0) || n < 0) return fail(ACCEL_E_INVALID, "bad argument");
    if (!little_endian()) return fail(ACCEL_E_UNSUPPORTED, "state files are little-endian");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(ACCEL_E_IO, std::string("cannot write ") + path);
    StateHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = 1;
    h.flags = loss_turn ? 1u : 0u;
    h.n = n;
    h.turn = turn;
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    if (ok && n > 0) ok = std::fwrite(r, sizeof(double) * 6, (size_t)n, f) == (size_t)n;
    if (ok && n > 0 && loss_turn) ok = std::fwrite(loss_turn, sizeof(int32_t), (size_t)n, f) == (size_t)n;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? ACCEL_OK : fail(ACCEL_E_IO, std::string("write failed: ") + path);
}

extern "C" int accel_state_read(const char* path, double** r, int64_t* n, int64_t* turn,
                                int32_t** loss_turn) {
    if (!path || !r || !n) return fail(ACCEL_E_INVALID, "NULL argument");
    *r = nullptr;
    if (loss_turn) *loss_turn = nullptr;
    if (!little_endian()) return fail(ACCEL_E_UNSUPPORTED, "state files are little-endian");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(ACCEL_E_IO, std::string("cannot open ") + path);
    StateHeader h{};
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, kMagic, 8) != 0 || h.version != 1 ||
        h.n < 0) {
        std::fclose(f);
        return fail(ACCEL_E_IO, std::string("not a particle-state file (version 1): ") + path);
    }
    // the particle count must match the file's length (also bounds the sizes computed from it)
    const int64_t per = (int64_t)sizeof(double) * 6 + ((h.flags & 1u) ? (int64_t)sizeof(int32_t) : 0);
    int64_t body = -1;
    if (std::fseek(f, 0, SEEK_END) == 0) {
        const long end = std::ftell(f);
        if (end >= (long)sizeof(h)) body = (int64_t)end - (int64_t)sizeof(h);
    }
    if (body < 0 || std::fseek(f, (long)sizeof(h), SEEK_SET) != 0 || h.n > body / per || h.n * per != body) {
        std::fclose(f);
        return fail(ACCEL_E_IO, std::string("particle-state file length does not match its particle count: ") + path);
    }
    double* rr = (double*)std::malloc(sizeof(double) * 6 * (size_t)std::max<int64_t>(1, h.n));
    int32_t* ll = (h.flags & 1u) ? (int32_t*)std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(1, h.n))
                                 : nullptr;
    bool ok = rr && (!(h.flags & 1u) || ll);
    if (ok && h.n > 0) ok = std::fread(rr, sizeof(double) * 6, (size_t)h.n, f) == (size_t)h.n;
    if (ok && ll && h.n > 0) ok = std::fread(ll, sizeof(int32_t), (size_t)h.n, f) == (size_t)h.n;
    std::fclose(f);
    if (!ok) {
        std::free(rr);
        std::free(ll);
        return fail(ACCEL_E_IO, std::string("particle-state file ends early: ") + path);
    }
    *r = rr;
    *n = h.n;
    if (turn) *turn = h.turn;
    if (loss_turn) *loss_turn = ll;
    else std::free(ll);
    return ACCEL_OK;
}

extern "C" void accel_state_free(void* p) { std::free(p); }
