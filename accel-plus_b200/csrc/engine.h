// engine.h — internal declarations shared by the host C++ and the CUDA translation units.
#pragma once
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>
#include <mutex>
#include <atomic>
#include <memory>
#include "accel_gpu.h"

namespace accel {

// ------------------------------------------------------------------------------------------
// Device element record.  One 384-byte record per element, 128-byte aligned, so an element
// spans exactly three L1/L2 lines.  Lines are "compiled" from accel_elem_desc on the host:
// every parameter-only expression the reference evaluates per particle (slice lengths, Yoshida
// weights, irho*tan(e), CRAD, ...) is evaluated once here with the reference's operation order,
// so the values are bit-identical to what the reference computes inside its loops.
// ------------------------------------------------------------------------------------------
enum DevOp : int32_t {
    OP_NOP = 0,        // Monitor, zero-length markers
    OP_DRIFT = 1,
    OP_STRMPOLE = 2,   // len > 0: Yoshida slices
    OP_STRKICK = 3,    // StrMPole with len == 0: one thin kick (accel.cpp:824-827)
    OP_BENDMPOLE = 4,
    OP_QUAD = 5,
    OP_BEND = 6,
    OP_CAVITY = 7,
    OP_APERTURE = 8,
    OP_CORRECTOR = 9,
    OP_MATRIX = 10,
    OP_SYNCRAD = 11,
    OP_TRANSWAKE = 12, // collective: never inside a fused range
    OP_LONGWAKE = 13,  // collective: never inside a fused range
    OP_CRABCAV = 14,
    OP_RFMULT = 15,
    OP_IDEALWIG = 16,
    OP_WIGTABLE = 17,
};

struct alignas(128) DevElem {
    int32_t op;
    int16_t nslice;
    int8_t order_eff;   // highest non-zero multipole index (exact Horner start for finite input)
    int8_t order_lit;   // the order the reference loops from (9 for StrMPole, MaxNPole-1 bends)
    int32_t flags;      // rad flag, on/off, skew-present bit (STR_SKEW)
    int32_t elem;       // element index in the line
    double h[14];       // hot payload: everything the fused kernel reads, in the first 128 B line
    double v[44];       // literal payload (plain kernel, tangent map, rare elements)
    double pad[4];
};
static_assert(sizeof(DevElem) == 512, "DevElem must be 512 bytes");
static_assert(offsetof(DevElem, v) == 128, "the hot payload must fill exactly the first line");

// hot payload slots (DevElem::h)
enum : int {
    H_LEN = 0,                                       // Drift, Cavity, Aperture
    H_L1 = 0, H_L2 = 1, H_K1 = 2, H_K2 = 3,          // StrMPole, BendMPole
    H_A = 4, H_B = 8,                                // StrMPole A[0..3], B[0..3]
    H_IRHO = 4, H_PSI1 = 5, H_PSI2 = 6, H_CRAD = 7,  // BendMPole
    H_BK1 = 8, H_BK2 = 9, H_BB = 10,                 // BendMPole K1, K2, B[0..3] at h[10..13]
    H_NV = 1, H_KZ = 2, H_PHIS = 3,                  // Cavity
    H_XMIN = 1, H_XMAX = 2, H_YMIN = 3, H_YMAX = 4,  // Aperture
};
constexpr int kHotOrder = 3;  // specialised multipole orders 0..3 read their coefficients from h

// payload slots
enum : int {
    V_LEN = 0,
    // StrMPole / BendMPole
    V_L1 = 1, V_L2 = 2, V_K1 = 3, V_K2 = 4, V_SL = 5,
    V_IRHO = 6, V_PSI1 = 7,
    V_A = 8,       // A[0..9] at v[8..17]
    V_B = 18,      // B[0..9] at v[18..27]
    V_PSI2 = 28, V_CRAD = 29, V_QECOEF = 30, V_BK1 = 31, V_BK2 = 32, V_ENERGY = 33,
    // Quad
    V_QK = 1,
    // Bend
    V_THETA = 1, V_GRD = 2, V_BIRHO = 3, V_BPSI1 = 4, V_BPSI2 = 5,
    // Cavity
    V_NV = 1, V_TF = 2, V_PHIS = 3, V_KZ = 4,
    // Aperture
    V_XMIN = 1, V_XMAX = 2, V_YMIN = 3, V_YMAX = 4,
    // Corrector
    V_KX = 1, V_KY = 2,
    // Matrix
    V_MAT = 8,     // 36 values v[8..43]
    // SyncRad
    V_ALFX = 1, V_ALFY = 2, V_ALFZ = 3, V_SX = 4, V_SY = 5, V_SZ = 6, V_SIGX = 7, V_SIGY = 8,
    V_SIGD = 9,
    // LongWake / TransWake keep their descriptor fields in v[1..12]
    V_W = 1,
    // CrabCav: devolt/energy, 2 pi f / c, phase, phase noise, voltage noise
    V_CNVX = 1, V_CNVY = 2, V_CK = 3, V_CPHIS = 4, V_CSIGPHI = 5, V_CSIGDVV = 6,
    // RFMult: 2 pi f / c, phase, phase noise, number of poles (A, B at V_A, V_B)
    V_RK = 1, V_RPHIS = 2, V_RSIGPHI = 3, V_RM = 4,
    // IdealWig: 2 pi / lambda, h, type, CGAMMA E^3 / (2 pi 1e9)
    V_WK = 1, V_WH = 2, V_WTYPE = 3, V_WCRAD = 4,
    // WigTable: grid sizes, device address of the table (bit pattern), registry id, len / 2
    V_TMX = 1, V_TMY = 2, V_TPTR = 3, V_TID = 4, V_THL = 5,
};

enum : int32_t { STR_SKEW = 1 << 8, STR_SKEW0 = 1 << 9 };  // any A non-zero; only A[0]

// ------------------------------------------------------------------------------------------
// Host-side error plumbing
// ------------------------------------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);

// lattice I/O (lattice_io.cpp)
int parse_lattice(const std::string& text, std::vector<accel_elem_desc>& out, std::string& err);
std::string format_lattice(const accel_elem_desc* e, int n, int precision);
void default_desc(int type, accel_elem_desc* d);
const char* type_name(int type);
int type_from_name(const std::string& s);

// WigTable kick tables (wigtable.cpp).  data = xl[mx], yl[my], xkick[my][mx], ykick[my][mx].
constexpr int kWigTabMaxX = 101, kWigTabMaxY = 21;  // MAX_WIGTAB_X / MAX_WIGTAB_Y, accel.h:401-402
struct WigTab {
    int mx = 0, my = 0;
    std::vector<double> data;
};
inline size_t wigtable_doubles(int mx, int my) { return (size_t)mx + my + 2 * (size_t)mx * my; }
std::shared_ptr<const WigTab> wigtable_find(int32_t id);
int wigtable_register(int mx, int my, const double* xl, const double* yl, const double* xkick,
                      const double* ykick, int32_t* id, std::string& err);

// compile descriptors to device records (compile.cpp)
int compile_line(const accel_elem_desc* d, int n, std::vector<DevElem>& out, std::string& err);
bool is_collective(int type);
bool is_supported(int type);
// Algorithmic flop count per particle-turn (model: add/sub/mul/div = 1 at the effective order)
double model_flops(const accel_elem_desc* d, int n);

}  // namespace accel
