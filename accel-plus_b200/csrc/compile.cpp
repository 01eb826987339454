// compile.cpp — lower accel_elem_desc descriptors to 512-byte device records (DevElem).
//
// Every expression below that depends only on element parameters is one the reference evaluates
// inside its per-particle loops; it is evaluated here once, with the same operands in the same
// order, so the doubles match the reference's bit for bit:
//   StrMPole  SL = len/nslice, L1 = SL*DRIFT1, ...          accel.cpp:803-808
//   BendMPole same, plus irho*tan(e1|e2)                     accel.cpp:652-656, atpass.cpp:192
//             CRAD = CGAMMA*E0^3/(TWOPI*1e9), uc_E0, QE coefficient   atpass.cpp:289-290,336
//   Cavity    nv = V/E, TWOPI*freq                           accel.cpp:905,919
//   Bend      irho*tan(e1|e2)                                accel.cpp:539-547
//   SyncRad   alf*, sqrt(2 alf*), sqrt(emit*beta)            accel.cpp:1808-1819
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include "engine.h"

namespace accel {

namespace {
const double PI_ = 3.1415926535897932384626;      // accel.h:23
const double TWOPI_ = 2 * PI_;                     // accel.h:24
const double C0_ = 2.99792458e8;                   // accel.h:29
const double CGAMMA_ = 8.846056192e-05;            // atpass.cpp:287
const double DRIFT1_ = 0.6756035959798286638;      // accel.h:44-47
const double DRIFT2_ = -0.1756035959798286639;
const double KICK1_ = 1.351207191959657328;
const double KICK2_ = -1.702414383919314656;
}  // namespace

bool is_collective(int type) { return type == ACCEL_TRANSWAKE || type == ACCEL_LONGWAKE; }

bool is_supported(int type) {
    switch (type) {
    case ACCEL_DRIFT: case ACCEL_QUAD: case ACCEL_CORRECTOR: case ACCEL_APERTURE:
    case ACCEL_MONITOR: case ACCEL_BEND: case ACCEL_BENDMPOLE: case ACCEL_STRMPOLE:
    case ACCEL_CAVITY: case ACCEL_TRANSWAKE: case ACCEL_MATRIX: case ACCEL_SYNCRAD:
    case ACCEL_LONGWAKE: case ACCEL_CRABCAV: case ACCEL_RFMULT: case ACCEL_IDEALWIG:
    case ACCEL_WIGTABLE:
        return true;
    default:
        return false;
    }
}

static int highest_nonzero(const double* a, const double* b, int upto) {
    int m = 0;
    for (int i = 0; i <= upto; i++)
        if ((a && a[i] != 0.0) || (b && b[i] != 0.0)) m = i;
    return m;
}

// Copy what the fused kernel reads into the first 128-byte line of the record.
static void fill_hot(DevElem& r) {
    for (int i = 0; i < 14; i++) r.h[i] = 0.0;
    switch (r.op) {
    case OP_DRIFT: r.h[H_LEN] = r.v[V_LEN]; break;
    case OP_STRMPOLE:
        r.h[H_L1] = r.v[V_L1]; r.h[H_L2] = r.v[V_L2]; r.h[H_K1] = r.v[V_K1]; r.h[H_K2] = r.v[V_K2];
        for (int i = 0; i <= kHotOrder; i++) { r.h[H_A + i] = r.v[V_A + i]; r.h[H_B + i] = r.v[V_B + i]; }
        break;
    case OP_BENDMPOLE:
        r.h[H_L1] = r.v[V_L1]; r.h[H_L2] = r.v[V_L2]; r.h[H_K1] = r.v[V_K1]; r.h[H_K2] = r.v[V_K2];
        r.h[H_IRHO] = r.v[V_IRHO]; r.h[H_PSI1] = r.v[V_PSI1]; r.h[H_PSI2] = r.v[V_PSI2];
        r.h[H_CRAD] = r.v[V_CRAD]; r.h[H_BK1] = r.v[V_BK1]; r.h[H_BK2] = r.v[V_BK2];
        for (int i = 0; i <= kHotOrder; i++) r.h[H_BB + i] = r.v[V_B + i];
        break;
    case OP_CAVITY:
        r.h[H_LEN] = r.v[V_LEN]; r.h[H_NV] = r.v[V_NV]; r.h[H_KZ] = r.v[V_KZ]; r.h[H_PHIS] = r.v[V_PHIS];
        break;
    case OP_APERTURE:
        r.h[H_LEN] = r.v[V_LEN];
        for (int i = 0; i < 4; i++) r.h[H_XMIN + i] = r.v[V_XMIN + i];
        break;
    default: break;
    }
}

int compile_line(const accel_elem_desc* d, int n, std::vector<DevElem>& out, std::string& err) {
    out.assign((size_t)n, DevElem{});
    for (int k = 0; k < n; k++) {
        const accel_elem_desc& e = d[k];
        DevElem& r = out[(size_t)k];
        std::memset(&r, 0, sizeof(r));
        r.elem = k;
        r.flags = e.flags;
        if (e.nslice > 32767) { err = "nslice above 32767"; return ACCEL_E_INVALID; }
        r.nslice = (int16_t)e.nslice;
        r.v[V_LEN] = e.len;
        switch (e.type) {
        case ACCEL_MONITOR:
            r.op = OP_NOP;
            break;
        case ACCEL_DRIFT:
            r.op = OP_DRIFT;
            break;
        case ACCEL_STRMPOLE: {
            if (e.len != 0 && e.nslice < 1) { err = "StrMPole nslice < 1"; return ACCEL_E_INVALID; }
            r.op = (e.len == 0) ? OP_STRKICK : OP_STRMPOLE;
            if (e.len != 0) {
                double SL = e.len / e.nslice;
                r.v[V_SL] = SL;
                r.v[V_L1] = SL * DRIFT1_;
                r.v[V_L2] = SL * DRIFT2_;
                r.v[V_K1] = SL * KICK1_;
                r.v[V_K2] = SL * KICK2_;
            }
            for (int i = 0; i < ACCEL_MAX_MPOLE; i++) {
                r.v[V_A + i] = e.poly_a[i];
                r.v[V_B + i] = e.poly_b[i];
            }
            r.order_lit = (int8_t)(ACCEL_MAX_MPOLE - 1);  // accel.cpp:826,837-841
            r.order_eff = (int8_t)highest_nonzero(e.poly_a, e.poly_b, ACCEL_MAX_MPOLE - 1);
            bool skew = false, skew_hi = false;
            for (int i = 0; i < ACCEL_MAX_MPOLE; i++) {
                skew |= (e.poly_a[i] != 0.0);
                if (i > 0) skew_hi |= (e.poly_a[i] != 0.0);
            }
            r.flags = skew ? (STR_SKEW | (skew_hi ? 0 : STR_SKEW0)) : 0;
            break;
        }
        case ACCEL_BENDMPOLE: {
            if (e.max_npole < 1 || e.max_npole > ACCEL_MAX_MPOLE) {
                err = std::string("BendMPole ") + e.famname + ": MaxNPole outside 1..10";
                return ACCEL_E_INVALID;
            }
            if (e.nslice < 1) { err = "BendMPole nslice < 1"; return ACCEL_E_INVALID; }
            r.op = OP_BENDMPOLE;
            double SL = e.len / e.nslice;
            r.v[V_SL] = SL;
            r.v[V_L1] = SL * DRIFT1_;
            r.v[V_L2] = SL * DRIFT2_;
            r.v[V_K1] = SL * KICK1_;
            r.v[V_K2] = SL * KICK2_;
            double irho = e.f[4];
            r.v[V_IRHO] = irho;
            r.v[V_PSI1] = irho * std::tan(e.f[1]);
            r.v[V_PSI2] = irho * std::tan(e.f[2]);
            double E0 = e.f[3];
            r.v[V_ENERGY] = E0;
            r.v[V_CRAD] = CGAMMA_ * E0 * E0 * E0 / (TWOPI_ * 1e9);
            double uc_E0 = 0.665 * E0 * E0 / 1.0e6 / 2.99792458E8 * std::fabs(irho) * 1000;
            r.v[V_QECOEF] = 55 * std::sqrt(3.0) / 72.0 * uc_E0;
            for (int i = 0; i < ACCEL_MAX_MPOLE; i++) r.v[V_B + i] = e.poly_b[i];
            r.order_lit = (int8_t)(e.max_npole - 1);
            r.order_eff = (int8_t)highest_nonzero(nullptr, e.poly_b, r.order_lit);
            r.v[V_BK1] = e.poly_b[1];                          // atpass.cpp:229 (read always)
            r.v[V_BK2] = (r.order_lit >= 2) ? e.poly_b[2] : 0;  // atpass.cpp:230-233
            r.flags = e.flags;                                  // radiation flag 0/1/2
            if (r.flags < 0 || r.flags > 2) r.flags = 0;
            break;
        }
        case ACCEL_QUAD:
            r.op = OP_QUAD;
            r.v[V_QK] = e.f[0];
            break;
        case ACCEL_BEND: {
            r.op = OP_BEND;
            r.v[V_THETA] = e.f[0];
            r.v[V_GRD] = e.f[3];
            r.v[V_BIRHO] = e.f[4];
            r.v[V_BPSI1] = e.f[4] * std::tan(e.f[1]);
            r.v[V_BPSI2] = e.f[4] * std::tan(e.f[2]);
            break;
        }
        case ACCEL_CAVITY: {
            r.op = OP_CAVITY;
            r.v[V_NV] = e.f[0] / e.f[3];
            r.v[V_TF] = TWOPI_ * e.f[1];
            r.v[V_PHIS] = e.f[2];
            r.v[V_KZ] = r.v[V_TF] / C0_;
            r.flags = e.flags ? 1 : 0;
            break;
        }
        case ACCEL_APERTURE:
            r.op = OP_APERTURE;
            for (int i = 0; i < 4; i++) r.v[V_XMIN + i] = e.f[i];
            break;
        case ACCEL_CORRECTOR:
            r.op = OP_CORRECTOR;
            r.v[V_KX] = e.f[0];
            r.v[V_KY] = e.f[1];
            break;
        case ACCEL_MATRIX:
            r.op = OP_MATRIX;
            for (int i = 0; i < 36; i++) r.v[V_MAT + i] = e.mat[i];
            break;
        case ACCEL_SYNCRAD: {
            r.op = OP_SYNCRAD;
            double energy = e.f[0], U0 = e.f[1], Jx = e.f[2], Jy = e.f[3];
            double Jz = 4 - Jx - Jy;
            double alfx = U0 / 2. / energy * Jx, alfy = U0 / 2. / energy * Jy,
                   alfz = U0 / 2. / energy * Jz;
            r.v[V_ALFX] = alfx; r.v[V_ALFY] = alfy; r.v[V_ALFZ] = alfz;
            r.v[V_SX] = std::sqrt(2. * alfx);
            r.v[V_SY] = std::sqrt(2. * alfy);
            r.v[V_SZ] = std::sqrt(2. * alfz);
            r.v[V_SIGX] = std::sqrt(e.f[4] * e.f[7]);
            r.v[V_SIGY] = std::sqrt(e.f[5] * e.f[8]);
            r.v[V_SIGD] = e.f[6];
            r.flags = e.flags & 3;
            break;
        }
        case ACCEL_CRABCAV:  // f: devoltx devolty freq phis energy sigphi sigdVV (accel.cpp:993-995)
            r.op = OP_CRABCAV;
            r.v[V_CNVX] = e.f[0] / e.f[4];
            r.v[V_CNVY] = e.f[1] / e.f[4];
            r.v[V_CK] = TWOPI_ * e.f[2] / C0_;
            r.v[V_CPHIS] = e.f[3];
            r.v[V_CSIGPHI] = e.f[5];
            r.v[V_CSIGDVV] = e.f[6];
            r.flags = e.flags ? 1 : 0;
            break;
        case ACCEL_RFMULT:  // f: freq phis energy sigphi sigdVV (accel.cpp:1148)
            r.op = OP_RFMULT;
            r.v[V_RK] = TWOPI_ * e.f[0] / C0_;
            r.v[V_RPHIS] = e.f[1];
            r.v[V_RSIGPHI] = e.f[3];
            r.v[V_RM] = e.max_npole;
            for (int i = 0; i < ACCEL_MAX_MPOLE; i++) { r.v[V_A + i] = e.poly_a[i]; r.v[V_B + i] = e.poly_b[i]; }
            break;
        case ACCEL_IDEALWIG: {  // f: lambda h wigtype energy (accel.cpp:1465, 1496)
            r.op = OP_IDEALWIG;
            r.v[V_WK] = 2.0 * PI_ / e.f[0];
            r.v[V_WH] = e.f[1];
            r.v[V_WTYPE] = e.f[2];
            const double en = e.f[3];
            r.v[V_WCRAD] = CGAMMA_ * en * en * en / (TWOPI_ * 1e9);
            r.flags = e.flags ? 1 : 0;
            break;
        }
        case ACCEL_WIGTABLE: {  // accel.cpp:1335-1377; the table's device address is set by the line
            const int32_t id = (int32_t)e.f[0];
            auto t = wigtable_find(id);
            if (!t) {
                err = std::string("WigTable ") + e.famname + ": no kick table with id " + std::to_string(id);
                return ACCEL_E_INVALID;
            }
            r.op = OP_WIGTABLE;
            r.v[V_TMX] = t->mx;
            r.v[V_TMY] = t->my;
            r.v[V_TID] = id;
            r.v[V_THL] = 0.5 * e.len;
            break;
        }
        case ACCEL_TRANSWAKE:
        case ACCEL_LONGWAKE:
            r.op = (e.type == ACCEL_TRANSWAKE) ? OP_TRANSWAKE : OP_LONGWAKE;
            for (int i = 0; i < 12; i++) r.v[V_W + i] = e.f[i];
            r.flags = e.flags ? 1 : 0;
            break;
        default:
            // parsed and kept (the line can be read, edited and written back); tracking through
            // it is refused by the C-ABI with ACCEL_E_UNSUPPORTED before any launch
            r.op = OP_NOP;
            break;
        }
        fill_hot(r);
    }
    return ACCEL_OK;
}

// Algorithmic flops per particle-turn at the effective multipole order (add/sub/mul/div = 1).
double model_flops(const accel_elem_desc* d, int n) {
    double f = 0;
    for (int k = 0; k < n; k++) {
        const accel_elem_desc& e = d[k];
        switch (e.type) {
        case ACCEL_DRIFT: f += 14; break;
        case ACCEL_STRMPOLE: {
            int m = highest_nonzero(e.poly_a, e.poly_b, ACCEL_MAX_MPOLE - 1);
            if (e.len == 0) f += 8 * m + 6;
            else f += e.nslice * (52.0 + 3.0 * (8 * m + 4));
            break;
        }
        case ACCEL_BENDMPOLE: {
            int m = highest_nonzero(nullptr, e.poly_b, e.max_npole - 1);
            double kick = (e.flags >= 1) ? (90.0 + 7 * m) : (44.0 + 7 * m);
            if (e.flags == 2) f += e.nslice * (2 * 46.0 + kick) + 8;
            else f += e.nslice * (4 * 46.0 + 3 * kick) + 8;
            break;
        }
        case ACCEL_QUAD: f += 60; break;
        case ACCEL_BEND: f += 98; break;
        case ACCEL_CAVITY: f += 6 + (e.len != 0 ? 28 : 0); break;
        case ACCEL_APERTURE: f += (e.len != 0 ? 14 : 0); break;
        case ACCEL_CORRECTOR: f += 4 + (e.len != 0 ? 28 : 0); break;
        case ACCEL_MATRIX: f += 66 + (e.len != 0 ? 28 : 0); break;
        case ACCEL_SYNCRAD: f += 6 + (e.len != 0 ? 28 : 0); break;
        case ACCEL_LONGWAKE: f += 8 + (e.len != 0 ? 28 : 0); break;
        case ACCEL_CRABCAV: f += 16 + (e.len != 0 ? 28 : 0); break;
        case ACCEL_RFMULT: f += 14 + 12 * e.max_npole + (e.len != 0 ? 28 : 0); break;
        case ACCEL_IDEALWIG: f += (e.len != 0 ? e.nslice * (28 + 12 + (e.flags ? 24 : 0)) : 0); break;
        // two cell coordinates (6) and two bilinear sums (2 x 13) per kick; two drifts per slice
        case ACCEL_WIGTABLE: f += (e.len != 0 ? e.nslice * (32 + 28 + 4) : 32); break;
        default: break;
        }
    }
    return f;
}

}  // namespace accel
