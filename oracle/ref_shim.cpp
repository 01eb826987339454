// ref_shim.cpp — test infrastructure only (the oracle).
//
// A C-callable shim over the reference Accel+ library (libaccel), compiled together with the
// reference's own sources by oracle/Makefile into oracle/_ref/libaccel_ref.so.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm load it, as the checker or
// the timed CPU baseline; the product never does.
//
// Every function forwards to the reference's public C++ API:
//   ALine::deserialize (aline.cpp:202), ALine::pass (aline.cpp:313-363), ALine::getm66
//   (aline.cpp:900-927), calctune/calcchrom/correctchrom (aline.cpp:1032,1108,1356),
//   setrfphase (aline.cpp:465), trackDA (aline.cpp:607), trackMA (aline.cpp:781),
//   set_*_onoff (aline.cpp:258,429,453), AStrMPole/ABendMPole setfield (accel.cpp:574-798),
//   trackDiffusion (aline.cpp:716), tracktune (aline.cpp:1159).
#include <fstream>
#include <string>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <omp.h>
#include "accel.h"
#include "matvec.h"
#include "utility.h"

namespace {
bool g_map_ready = false;
void ensure_map() {
    if (!g_map_ready) { AccelElement::initializemap(); g_map_ready = true; }
}
ALine* L(void* h) { return static_cast<ALine*>(h); }
}  // namespace

extern "C" {

void* ref_line_load(const char* path) {
    ensure_map();
    std::ifstream fin(path);
    if (!fin.good()) return nullptr;
    return ALine::deserialize(fin);
}

void ref_line_free(void* h) { delete L(h); }

int ref_line_nelem(void* h) { return (int)L(h)->getnumber(); }

void ref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }

int ref_max_threads(void) { return omp_get_max_threads(); }

// ALine::pass(r, N, nturn): the OpenMP-by-line turn loop.
void ref_pass(void* h, double* r, int N, int nturn) { L(h)->pass(r, N, nturn); }

// ALine::pass(r, N, st, ed): one pass through elements [st, ed).
void ref_pass_range(void* h, double* r, int N, int st, int ed) {
    L(h)->pass(r, N, (unsigned)st, (unsigned)ed);
}

// Per-turn NaN scan, as trackDA's loss-turn branch does (aline.cpp:646-659), except that
// survivors get -1 so a loss in turn 0 is distinguishable from survival.
void ref_track_loss(void* h, double* r, int N, int nturn, int* loss_turn) {
    for (int i = 0; i < N; i++) loss_turn[i] = -1;
    for (int t = 0; t < nturn; t++) {
        L(h)->pass(r, N);
        for (int i = 0; i < N; i++)
            if (loss_turn[i] < 0 && std::isnan(r[6 * i])) loss_turn[i] = t;
    }
}

// The same scan, also keeping in last[6N] each particle's state at the end of the last turn it
// survived (the final state for survivors): how far perturbed runs are apart just before a loss.
void ref_track_loss_last(void* h, double* r, int N, int nturn, int* loss_turn, double* last) {
    for (int i = 0; i < N; i++) loss_turn[i] = -1;
    for (int i = 0; i < 6 * N; i++) last[i] = r[i];
    for (int t = 0; t < nturn; t++) {
        L(h)->pass(r, N);
        for (int i = 0; i < N; i++) {
            if (loss_turn[i] >= 0) continue;
            if (std::isnan(r[6 * i])) loss_turn[i] = t;
            else
                for (int k = 0; k < 6; k++) last[6 * i + k] = r[6 * i + k];
        }
    }
}

void ref_m66(void* h, int st, int ed, double dpp, double delta, double* m36) {
    Mat m(6, 6);
    L(h)->getm66(m, (unsigned)st, (unsigned)ed, dpp, delta);
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) m36[6 * i + j] = m[i + 1][j + 1];
}

void ref_calc_tune(void* h, double* nux, double* nuy) { L(h)->calctune(*nux, *nuy); }

void ref_calc_chrom(void* h, double* cx, double* cy) { L(h)->calcchrom(*cx, *cy); }

static unsigned fam_list(void* h, const char* type, const char* fam, unsigned* list) {
    return L(h)->findelements(list, std::string(type), std::string(fam), 0);
}

// correct_chrom deck command (process.cpp:658-767): two families, 2x2 FD response, one step.
void ref_correct_chrom(void* h, const char* type, const char* fam1, const char* fam2,
                       double* cx, double* cy) {
    static unsigned l1[MAX_ELEMENT], l2[MAX_ELEMENT];
    unsigned n1 = fam_list(h, type, fam1, l1), n2 = fam_list(h, type, fam2, l2);
    if (!n1 || !n2) return;
    L(h)->correctchrom(*cx, *cy, n1, n2, l1, l2);
}

void ref_correct_tune(void* h, const char* type, const char* fam1, const char* fam2,
                      double* nux, double* nuy) {
    static unsigned l1[MAX_ELEMENT], l2[MAX_ELEMENT];
    unsigned n1 = fam_list(h, type, fam1, l1), n2 = fam_list(h, type, fam2, l2);
    if (!n1 || !n2) return;
    L(h)->correcttune(*nux, *nuy, n1, n2, l1, l2);
}

double ref_setrfphase(void* h) { return L(h)->setrfphase(); }

void ref_set_rad(void* h, int flag) { L(h)->set_rad_onoff((unsigned)flag); }
void ref_set_cavity(void* h, int on) { L(h)->set_cavity_onoff(on != 0); }
void ref_set_wake(void* h, int on) { L(h)->set_wake_onoff(on != 0); }
void ref_set_crab(void* h, int on) { L(h)->set_crab_onoff(on != 0); }
void ref_set_energy(void* h, double en) { L(h)->setenergy(en); }

// PolynomB/PolynomA[index] of a StrMPole (accel.cpp:773-785) or PolynomB of a BendMPole.
int ref_set_poly(void* h, int idx, int is_a, int index, double v) {
    AccelElement* e = L(h)->getelement((unsigned)idx);
    if (!e) return -1;
    const char* f = is_a ? "PolynomA" : "PolynomB";
    if (e->gettype() == "StrMPole") { ((AStrMPole*)e)->setfield(&v, f, (unsigned)index); return 0; }
    if (e->gettype() == "BendMPole" && !is_a) { ((ABendMPole*)e)->setfield(&v, f, (unsigned)index); return 0; }
    return -1;
}

int ref_get_poly(void* h, int idx, int is_a, int index, double* v) {
    AccelElement* e = L(h)->getelement((unsigned)idx);
    if (!e) return -1;
    const char* f = is_a ? "PolynomA" : "PolynomB";
    if (e->gettype() == "StrMPole") { ((AStrMPole*)e)->getfield(v, f, (unsigned)index); return 0; }
    if (e->gettype() == "BendMPole" && !is_a) { ((ABendMPole*)e)->getfield(v, f, (unsigned)index); return 0; }
    return -1;
}

int ref_set_double_field(void* h, int idx, const char* name, double v) {
    AccelElement* e = L(h)->getelement((unsigned)idx);
    if (!e) return -1;
    e->setfield(&v, std::string(name));
    return 0;
}

int ref_get_double_field(void* h, int idx, const char* name, double* v) {
    AccelElement* e = L(h)->getelement((unsigned)idx);
    if (!e) return -1;
    e->getfield(v, std::string(name));
    return 0;
}

int ref_set_nslice(void* h, int idx, int ns) {
    AccelElement* e = L(h)->getelement((unsigned)idx);
    if (!e) return -1;
    e->setfield(&ns, std::string("NSlice"));
    return 0;
}

void ref_srand(unsigned seed) { srand(seed); }

double ref_grandn(void) { return grandn(0.0, 1.0); }

double ref_naff(int n, double* data, double xlow, double xhi) { return naff(n, data, xlow, xhi); }

double ref_trackDA(void* h, double xmax, double xmin, double ymax, int nturn, int nray,
                   int nstep, double* rx, double* ry) {
    return L(h)->trackDA(xmax, xmin, ymax, nturn, (unsigned)nray, nstep, rx, ry, false);
}

// trackMA over the elements listed in lfam (aline.cpp:781-836).
double ref_trackMA(void* h, double dppmax, double dppmin, int nturn, int nstep,
                   double* dpp_plus, double* dpp_minus, int nfam, const int* lfam) {
    unsigned* l = new unsigned[nfam > 0 ? nfam : 1];
    for (int i = 0; i < nfam; i++) l[i] = (unsigned)lfam[i];
    double v = L(h)->trackMA(dppmax, dppmin, nturn, (unsigned)nstep, dpp_plus, dpp_minus,
                             (unsigned)nfam, l);
    delete[] l;
    return v;
}

// Tune diffusion (aline.cpp:716-779) and tracked tunes (aline.cpp:1159-1186).
double ref_trackDiffusion(void* h, int nturn, int np, double* x0, double* y0, double* nux, double* nuy,
                          double* dif, double xlow, double xhi, double ylow, double yhi) {
    return L(h)->trackDiffusion(nturn, (unsigned)np, x0, y0, nux, nuy, dif, xlow, xhi, ylow, yhi);
}

void ref_tracktune(void* h, int nturn, double x0, double y0, double xlow, double xhi, double ylow,
                   double yhi, double* tunex, double* tuney) {
    L(h)->tracktune(*tunex, *tuney, (unsigned)nturn, x0, y0, xlow, xhi, ylow, yhi);
}

// Beam moments (utility.cpp:387-438).
int ref_beam_stat(double* r, int N, double* mean, double* sigma, double* cross) {
    return calc_beam_stat(r, N, mean, sigma, cross);
}

// Closed orbit (aline.cpp:838-889); six doubles out (four for the 4D form).
void ref_getco4(void* h, double dp, double* rc) {
    Vec v(4);
    L(h)->getco4(v, dp);
    for (int i = 0; i < 4; i++) rc[i] = v[i + 1];
}

}  // extern "C"
