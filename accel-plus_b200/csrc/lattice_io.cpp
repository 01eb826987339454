// lattice_io.cpp — the Accel+ lattice text format, read and written on the host.
//
// Reading follows AccelElement::deserialize (reference src/lib/accel/accel.cpp:67-133): a family
// name token (with or without a trailing ':'; without one, input is skipped to the next ':'),
// then a type name from the type registry (accel.cpp:25-43), then the type's parameters as the
// per-type create() readers take them:
//   Drift      len                                   accel.cpp:147-157
//   Quad       len K                                 accel.cpp:184-192
//   Corrector  len kickx kicky                       accel.cpp:236-244
//   Aperture   len xmin xmax ymin ymax               accel.cpp:299-307
//   Monitor    len interval ratio                    accel.cpp:394-407
//   Bend       len theta e1 e2 K                     accel.cpp:481-489
//   BendMPole  len theta e1 e2 MaxNPole / PolyB...   accel.cpp:560-573
//   StrMPole   len MaxNPole / PolyB... / PolyA...    accel.cpp:718-736
//   Cavity     len volt freq phis energy             accel.cpp:860-869
//   CrabCav    len dvx dvy freq phis en sigphi sigdVV accel.cpp:937-946
//   RFMult     len freq phis en sigphi sigdVV MaxNPole / PolyB / PolyA   accel.cpp:1058-1072
//   WigTable   len nslice mx my / xl / yl / xkick rows / blank / ykick rows accel.cpp:1294-1333
//              (the numbers after the size line are read as one sequence, so the blank line
//              is optional; the table goes to the registry, the descriptor keeps its id)
//   IdealWig   len nslice lambda h wigtype           accel.cpp:1449-1461
//   TransWake  len energy Ne Wx fRx Qx Wy fRy Qy     accel.cpp:1546-1554
//   Matrix     len / six rows of six                 accel.cpp:1673-1687
//   SyncRad    len en U0 Jx Jy / emitx emity sigdpp betax betay  accel.cpp:1743-1753
//   LongWake   len energy charge Rs fr Q nbins       (no reference counterpart)
// "RETURN" ends the line (accel.cpp:82-84).  Differences, all on malformed input: a '!' token
// comments out the rest of its line (the reference skips the line and then reuses the '!' token
// as the next element's family name), a missing number takes the type's default (the reference
// keeps the previous element's value), and an unknown type or a MaxNPole outside 1..10 is an
// error (the reference stops reading, or overruns its arrays).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>
#include "engine.h"

namespace accel {

namespace {
const double kPi = 3.1415926535897932384626;  // reference PI, accel.h:23

struct Cursor {
    const std::string& s;
    size_t p = 0;
    explicit Cursor(const std::string& str) : s(str) {}
    bool eof() const { return p >= s.size(); }
    void skip_ws() { while (p < s.size() && std::isspace((unsigned char)s[p])) p++; }
    bool token(std::string& out) {
        skip_ws();
        if (eof()) return false;
        size_t b = p;
        while (p < s.size() && !std::isspace((unsigned char)s[p])) p++;
        out = s.substr(b, p - b);
        return true;
    }
    std::string rest_of_line() {
        size_t b = p;
        while (p < s.size() && s[p] != '\n') p++;
        std::string r = s.substr(b, p - b);
        if (p < s.size()) p++;
        return r;
    }
    bool skip_to(char c) {
        while (p < s.size() && s[p] != c) p++;
        if (p >= s.size()) return false;
        p++;
        return true;
    }
    bool number(double& v) {
        std::string t;
        size_t save = p;
        if (!token(t)) return false;
        char* end = nullptr;
        v = std::strtod(t.c_str(), &end);
        if (end == t.c_str()) { p = save; return false; }
        return true;
    }
};

// Parse up to n numbers from one line; returns how many were read.
int line_numbers(const std::string& line, double* v, int n) {
    std::istringstream is(line);
    int k = 0;
    std::string t;
    while (k < n && (is >> t)) {
        char* end = nullptr;
        double x = std::strtod(t.c_str(), &end);
        if (end == t.c_str()) break;
        v[k++] = x;
    }
    return k;
}
}  // namespace

const char* type_name(int type) {
    switch (type) {
    case ACCEL_DRIFT: return "Drift";
    case ACCEL_QUAD: return "Quad";
    case ACCEL_CORRECTOR: return "Corrector";
    case ACCEL_APERTURE: return "Aperture";
    case ACCEL_MONITOR: return "Monitor";
    case ACCEL_BEND: return "Bend";
    case ACCEL_BENDMPOLE: return "BendMPole";
    case ACCEL_STRMPOLE: return "StrMPole";
    case ACCEL_CAVITY: return "Cavity";
    case ACCEL_WIGTABLE: return "WigTable";
    case ACCEL_IDEALWIG: return "IdealWig";
    case ACCEL_CRABCAV: return "CrabCav";
    case ACCEL_RFMULT: return "RFMult";
    case ACCEL_TRANSWAKE: return "TransWake";
    case ACCEL_MATRIX: return "Matrix";
    case ACCEL_SYNCRAD: return "SyncRad";
    case ACCEL_LONGWAKE: return "LongWake";
    default: return "undefined";
    }
}

int type_from_name(const std::string& s) {
    for (int t = ACCEL_DRIFT; t <= ACCEL_LONGWAKE; t++)
        if (s == type_name(t)) return t;
    return 0;
}

// The reference constructors' defaults (accel.h:79-570).
void default_desc(int type, accel_elem_desc* d) {
    std::memset(d, 0, sizeof(*d));
    d->type = type;
    d->nslice = 1;
    std::snprintf(d->famname, sizeof(d->famname), "undefined");
    switch (type) {
    case ACCEL_APERTURE: d->f[0] = -1.0; d->f[1] = 1.0; d->f[2] = -1.0; d->f[3] = 1.0; break;
    case ACCEL_MONITOR: d->f[0] = 1; d->f[1] = 1.0; break;
    case ACCEL_BENDMPOLE: d->nslice = 10; d->f[3] = 3000; d->max_npole = ACCEL_MAX_MPOLE; break;
    case ACCEL_STRMPOLE: d->nslice = 10; d->max_npole = ACCEL_MAX_MPOLE; break;
    case ACCEL_CAVITY: d->f[1] = 476.314e6; d->f[3] = 3000; d->flags = 1; break;
    case ACCEL_CRABCAV: d->f[2] = 476.314e6 * 6; d->f[4] = 3000; break;
    case ACCEL_RFMULT: d->f[0] = 476.314e6 * 6; d->f[2] = 3000; break;
    case ACCEL_IDEALWIG: d->f[0] = 0.10; d->f[3] = 3000; break;  // f3: energy (not in the file)
    case ACCEL_TRANSWAKE:
        d->f[0] = 3000; d->f[3] = 1.0e10; d->f[4] = 1; d->f[6] = 1.0e10; d->f[7] = 1; break;
    case ACCEL_MATRIX:
        for (int i = 0; i < 6; i++) d->mat[6 * i + i] = 1.0;
        break;
    case ACCEL_SYNCRAD:
        d->f[0] = 3000; d->f[1] = 0.881; d->f[2] = 1.35; d->f[3] = 1; d->f[4] = 1e-9;
        d->f[5] = 10e-12; d->f[6] = 0.001; d->f[7] = 1; d->f[8] = 1;
        break;
    case ACCEL_LONGWAKE: d->f[0] = 3000; d->f[4] = 1; d->f[5] = 256; break;
    default: break;
    }
}

int parse_lattice(const std::string& text, std::vector<accel_elem_desc>& out, std::string& err) {
    Cursor c(text);
    out.clear();
    std::string fam, type;
    for (;;) {
        if (!c.token(fam)) break;
        if (fam == "RETURN") break;
        if (fam[0] == '!') { c.rest_of_line(); continue; }
        if (fam.back() == ':') fam.pop_back();
        else if (!c.skip_to(':')) break;
        if (!c.token(type)) break;
        int t = type_from_name(type);
        if (!t) { err = "type not found: " + type; return ACCEL_E_IO; }
        accel_elem_desc d;
        default_desc(t, &d);
        std::snprintf(d.famname, sizeof(d.famname), "%s", fam.c_str());
        double v[16] = {0};
        std::string line = c.rest_of_line();
        int k = line_numbers(line, v, 16);
        auto get = [&](int i, double dflt) { return i < k ? v[i] : dflt; };
        d.len = get(0, 0.0);
        switch (t) {
        case ACCEL_DRIFT: break;
        case ACCEL_QUAD: d.f[0] = get(1, 0.0); break;
        case ACCEL_CORRECTOR: d.f[0] = get(1, 0.0); d.f[1] = get(2, 0.0); break;
        case ACCEL_APERTURE:
            for (int i = 0; i < 4; i++) d.f[i] = get(1 + i, d.f[i]);
            break;
        case ACCEL_MONITOR: {  // accel.cpp:398-405 clamps
            d.len = 0;
            double it = get(1, 1), ra = get(2, 1.0);
            if (it <= 1) it = 1;
            if (ra < 0) ra = 0.1;
            if (ra > 1.0) ra = 1.0;
            d.f[0] = it; d.f[1] = ra;
            break;
        }
        case ACCEL_BEND:
            d.f[0] = get(1, 0); d.f[1] = get(2, 0); d.f[2] = get(3, 0); d.f[3] = get(4, 0);
            d.f[4] = d.f[0] / d.len;  // irho = theta/len, accel.h:170
            break;
        case ACCEL_BENDMPOLE: {
            d.f[0] = get(1, 0); d.f[1] = get(2, 0); d.f[2] = get(3, 0);
            d.max_npole = (int)get(4, ACCEL_MAX_MPOLE);
            d.f[4] = d.f[0] / d.len;
            if (d.max_npole < 1 || d.max_npole > ACCEL_MAX_MPOLE) {
                err = std::string("BendMPole ") + d.famname + ": MaxNPole outside 1..10";
                return ACCEL_E_IO;
            }
            for (int i = 0; i < d.max_npole; i++) c.number(d.poly_b[i]);
            c.rest_of_line();
            break;
        }
        case ACCEL_STRMPOLE: {
            d.max_npole = (int)get(1, ACCEL_MAX_MPOLE);
            if (d.max_npole < 0 || d.max_npole > ACCEL_MAX_MPOLE) {
                err = std::string("StrMPole ") + d.famname + ": MaxNPole outside 0..10";
                return ACCEL_E_IO;
            }
            for (int i = 0; i < d.max_npole; i++) c.number(d.poly_b[i]);
            c.rest_of_line();
            for (int i = 0; i < d.max_npole; i++) c.number(d.poly_a[i]);
            c.rest_of_line();
            break;
        }
        case ACCEL_CAVITY:
            d.f[0] = get(1, 0); d.f[1] = get(2, 0); d.f[2] = get(3, 0); d.f[3] = get(4, 3000);
            d.flags = 1;  // ACavity ctor: flag_onoff = true
            break;
        case ACCEL_CRABCAV:
            for (int i = 0; i < 7; i++) d.f[i] = get(1 + i, d.f[i]);
            break;
        case ACCEL_RFMULT: {
            for (int i = 0; i < 5; i++) d.f[i] = get(1 + i, d.f[i]);
            d.max_npole = (int)get(6, 0);
            if (d.max_npole < 0 || d.max_npole > ACCEL_MAX_MPOLE) { err = "RFMult MaxNPole"; return ACCEL_E_IO; }
            for (int i = 0; i < d.max_npole; i++) c.number(d.poly_b[i]);
            c.rest_of_line();
            for (int i = 0; i < d.max_npole; i++) c.number(d.poly_a[i]);
            c.rest_of_line();
            break;
        }
        case ACCEL_WIGTABLE: {  // the table is registered; the descriptor keeps its id
            d.nslice = (int)get(1, 1);
            const int mx = (int)get(2, 0), my = (int)get(3, 0);
            if (mx < 2 || mx > kWigTabMaxX || my < 2 || my > kWigTabMaxY) {
                err = std::string("WigTable ") + d.famname + ": table size outside 2..101 x 2..21";
                return ACCEL_E_IO;
            }
            std::vector<double> t(wigtable_doubles(mx, my));
            for (size_t i = 0; i < t.size(); i++)
                if (!c.number(t[i])) {
                    err = std::string("WigTable ") + d.famname + ": table ends early";
                    return ACCEL_E_IO;
                }
            c.rest_of_line();
            int32_t id = 0;
            const double* p = t.data();
            int st = wigtable_register(mx, my, p, p + mx, p + mx + my, p + mx + my + mx * my, &id, err);
            if (st) { err = std::string("WigTable ") + d.famname + ": " + err; return ACCEL_E_IO; }
            d.f[0] = id;
            break;
        }
        case ACCEL_IDEALWIG:
            d.nslice = (int)get(1, 1); d.f[0] = get(2, 0.10); d.f[1] = get(3, 0); d.f[2] = get(4, 0);
            break;
        case ACCEL_TRANSWAKE:
            for (int i = 0; i < 8; i++) d.f[i] = get(1 + i, d.f[i]);
            break;
        case ACCEL_MATRIX:
            for (int i = 0; i < 6; i++) {
                std::string row = c.rest_of_line();
                double m[6] = {0, 0, 0, 0, 0, 0};
                line_numbers(row, m, 6);
                for (int j = 0; j < 6; j++) d.mat[6 * i + j] = m[j];
            }
            break;
        case ACCEL_SYNCRAD: {
            d.f[0] = get(1, d.f[0]); d.f[1] = get(2, d.f[1]); d.f[2] = get(3, d.f[2]); d.f[3] = get(4, d.f[3]);
            std::string l2 = c.rest_of_line();
            double w[5] = {d.f[4], d.f[5], d.f[6], d.f[7], d.f[8]};
            line_numbers(l2, w, 5);
            for (int i = 0; i < 5; i++) d.f[4 + i] = w[i];
            break;
        }
        case ACCEL_LONGWAKE:
            for (int i = 0; i < 6; i++) d.f[i] = get(1 + i, d.f[i]);
            break;
        default: break;
        }
        out.push_back(d);
    }
    return ACCEL_OK;
}

// The reference's serialize() layout (accel.cpp:143-1742), with a caller-chosen precision so
// that a written lattice reads back bit-identically at precision 17.  As in the reference, the
// frequency and phase of Cavity, CrabCav and RFMult are written with at least 16 digits
// (accel.cpp:855, 932, 1047).
std::string format_lattice(const accel_elem_desc* e, int n, int precision) {
    std::string s;
    char buf[256];
    auto num = [&](double x) {
        std::snprintf(buf, sizeof(buf), "%.*g", precision, x);
        s += buf;
    };
    auto num16 = [&](double x) {
        std::snprintf(buf, sizeof(buf), "%.*g", precision > 16 ? precision : 16, x);
        s += buf;
    };
    auto tab = [&]() { s += "\t"; };
    for (int k = 0; k < n; k++) {
        const accel_elem_desc& d = e[k];
        s += d.famname;
        s += "  : \t";
        s += type_name(d.type);
        tab();
        num(d.len);
        switch (d.type) {
        case ACCEL_QUAD: tab(); num(d.f[0]); break;
        case ACCEL_CORRECTOR: tab(); num(d.f[0]); tab(); num(d.f[1]); break;
        case ACCEL_APERTURE: for (int i = 0; i < 4; i++) { tab(); num(d.f[i]); } break;
        case ACCEL_MONITOR: tab(); num(d.f[0]); tab(); num(d.f[1]); break;
        case ACCEL_BEND: for (int i = 0; i < 4; i++) { tab(); num(d.f[i]); } break;
        case ACCEL_BENDMPOLE:
            for (int i = 0; i < 3; i++) { tab(); num(d.f[i]); }
            tab(); s += std::to_string(d.max_npole);
            s += "\n\t\t\t";
            for (int i = 0; i < d.max_npole; i++) { num(d.poly_b[i]); tab(); }
            break;
        case ACCEL_STRMPOLE:
            tab(); s += std::to_string(d.max_npole);
            s += "\n\t\t\t";
            for (int i = 0; i < d.max_npole; i++) { num(d.poly_b[i]); tab(); }
            s += "\n\t\t\t";
            for (int i = 0; i < d.max_npole; i++) { num(d.poly_a[i]); tab(); }
            break;
        case ACCEL_CAVITY:
            for (int i = 0; i < 4; i++) { tab(); (i == 1 || i == 2) ? num16(d.f[i]) : num(d.f[i]); }
            break;
        case ACCEL_CRABCAV:
            for (int i = 0; i < 7; i++) { tab(); (i == 2 || i == 3) ? num16(d.f[i]) : num(d.f[i]); }
            break;
        case ACCEL_RFMULT:
            for (int i = 0; i < 5; i++) { tab(); i < 2 ? num16(d.f[i]) : num(d.f[i]); }
            tab(); s += std::to_string(d.max_npole);
            s += "\n\t\t\t";
            for (int i = 0; i < d.max_npole; i++) { num(d.poly_b[i]); tab(); }
            s += "\n\t\t\t";
            for (int i = 0; i < d.max_npole; i++) { num(d.poly_a[i]); tab(); }
            break;
        case ACCEL_IDEALWIG:
            tab(); s += std::to_string(d.nslice);
            for (int i = 0; i < 3; i++) { tab(); num(d.f[i]); }
            break;
        case ACCEL_WIGTABLE: {  // accel.cpp:1247-1270: sizes, xl, yl, xkick rows, blank, ykick rows
            auto t = wigtable_find((int32_t)d.f[0]);
            const int mx = t ? t->mx : 0, my = t ? t->my : 0;
            tab(); s += std::to_string(d.nslice);
            tab(); s += std::to_string(mx);
            tab(); s += std::to_string(my);
            if (!t) break;
            const double* p = t->data.data();
            s += "\n";
            for (int j = 0; j < mx; j++) { num(p[j]); tab(); }
            s += "\n";
            for (int i = 0; i < my; i++) { num(p[mx + i]); tab(); }
            for (int k = 0; k < 2; k++) {
                const double* z = p + mx + my + (size_t)k * mx * my;
                if (k == 1) s += "\n";
                for (int i = 0; i < my; i++) {
                    s += "\n";
                    for (int j = 0; j < mx; j++) { num(z[i * mx + j]); tab(); }
                }
            }
            break;
        }
        case ACCEL_TRANSWAKE: for (int i = 0; i < 8; i++) { tab(); num(d.f[i]); } break;
        case ACCEL_MATRIX:
            for (int i = 0; i < 6; i++) {
                s += "\n\t";
                for (int j = 0; j < 6; j++) { num(d.mat[6 * i + j]); tab(); }
            }
            break;
        case ACCEL_SYNCRAD:
            for (int i = 0; i < 4; i++) { tab(); num(d.f[i]); }
            s += "\n\t";
            for (int i = 4; i < 9; i++) { num(d.f[i]); tab(); }
            break;
        case ACCEL_LONGWAKE: for (int i = 0; i < 6; i++) { tab(); num(d.f[i]); } break;
        default: break;
        }
        s += "\n";
    }
    (void)kPi;
    return s;
}

}  // namespace accel
