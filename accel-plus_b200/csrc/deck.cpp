// deck.cpp — `accel+gpu`: the reference's input-deck interpreter (src/process.cpp) over the GPU.
//
//   accel+gpu DECK [--device N] [--plain | --exact] [--seed S]
//
// Blocks (process.cpp:40-107): Lattice, Optics, Track, DAMA, each ended by `End`; Survey is
// accepted and ignored; STOP / RETURN end the deck.  Lines: '#' and '%' start comments, a trailing
// '\' continues a line (mgetline, process.cpp:117-135); block and command keywords match
// case-insensitively by prefix (lookforblock, process.cpp:136-160).  Commands:
//   Lattice  file_name = F[, type=ERING]  reset_first  print_elem_value  print_lat_summary
//            export_element  correct_tune  correct_chrom (both add EXACT for Newton iterations
//            on exact one-turn matrices)  set_max_num_threads  modify_element  set_flags
//   Optics   print_tune  print_chrom  print_matrix  print_optics
//   Track    Distribution (none | Zero NPar= | Coordinate r=(..;..) | Gaussian .. | Linear ..
//            | Load F[, format=plain|accel-export|binary]; shift=(..); Print)  Monitor
//            Do_Track (+ save=F: a lossless binary checkpoint of the final distribution)  Transport
//   DAMA     track_DA  track_MA  track_dNudJ
// Differences: Gaussian distributions come from a seeded generator (--seed; the reference seeds
// rand() with the time, process.cpp:42); a family member picked with index >= 2 is that member
// (the reference's findelements leaves list[0] unset then, aline.cpp:531-533); apply_setpt is
// reported as not supported.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <memory>
#include <random>
#include <regex>
#include <sstream>
#include <string>
#include <vector>
#include "accel_gpu.h"
#include "host_aline.hpp"

using accelgpu::ALine;
using std::cout;
using std::endl;
using std::string;

namespace {

string upper(string s) {
    for (auto& c : s) c = (char)std::toupper((unsigned char)c);
    return s;
}
bool iequal(const string& a, const string& b) { return upper(a) == upper(b); }
void trim(string& s) {
    size_t a = s.find_first_not_of(" \t\r\n\f\v");
    size_t b = s.find_last_not_of(" \t\r\n\f\v");
    s = (a == string::npos) ? string() : s.substr(a, b - a + 1);
}
void strip_comment(string& s) {
    size_t p = s.find_first_of("#%");
    if (p != string::npos) s.erase(p);
}

bool mgetline(std::istream& in, string& line) {
    if (!std::getline(in, line)) return false;
    strip_comment(line);
    while (!line.empty() && std::isspace((unsigned char)line.back())) line.pop_back();
    while (!line.empty() && line.back() == '\\') {
        line.back() = ' ';
        string nl;
        if (!std::getline(in, nl)) break;
        strip_comment(nl);
        while (!nl.empty() && std::isspace((unsigned char)nl.back())) nl.pop_back();
        line += nl;
    }
    return true;
}

// returns the index of the matched key, -1 at end of input or STOP/RETURN
int lookfor(std::istream& in, string& matched, const std::vector<string>& keys) {
    string line;
    while (mgetline(in, line)) {
        trim(line);
        if (line.empty()) continue;
        string u = upper(line);
        if (u == "STOP" || u == "RETURN") return -1;
        for (size_t i = 0; i < keys.size(); i++)
            if (u.compare(0, keys[i].size(), keys[i]) == 0) {
                matched = line;
                return (int)i;
            }
    }
    return -1;
}

// "key=value" pairs after the command's first ':' or '='; commas or blanks separate them and a
// value may be a bracketed group: "nturn=100, radiation = off" or "r=(1,0,0,0,0,0;2,0,0,0,0,0)".
// Words without '=' come back with an empty value.
std::vector<std::pair<string, string>> kv(string s) {
    size_t p = s.find_first_of(":=");
    s = (p == string::npos) ? string() : s.substr(p + 1);
    static const std::regex tok(R"(([A-Za-z_][A-Za-z0-9_\[\]]*)\s*(=\s*(\([^)]*\)|\[[^\]]*\]|[^\s,]+))?)");
    std::vector<std::pair<string, string>> out;
    for (auto it = std::sregex_iterator(s.begin(), s.end(), tok); it != std::sregex_iterator(); ++it)
        out.push_back({upper((*it)[1].str()), (*it)[3].str()});
    return out;
}

string get(const std::vector<std::pair<string, string>>& a, const string& k, const string& dflt = "") {
    for (auto& p : a)
        if (p.first == k) return p.second;
    return dflt;
}
bool has(const std::vector<std::pair<string, string>>& a, const string& k) {
    for (auto& p : a)
        if (p.first == k) return true;
    return false;
}

string now() {
    time_t t = time(nullptr);
    char b[64];
    strftime(b, sizeof(b), "UTC %Y-%m-%d %X", localtime(&t));
    return b;
}

// element selection as get_elem_list (process.cpp:1050-1100): no type -> the element `index`;
// ALL -> every element; type only -> all of the type, or its index-th (1-based); type + famname
// -> findelements, optionally narrowed by an index list "[i j k]" (entries 1 .. n-1).
std::vector<unsigned> select(ALine& L, const string& type, const string& fam, unsigned index,
                             const string& indices = "") {
    std::vector<unsigned> list(L.getnumber() + 1);
    unsigned n = 0;
    if (type.empty()) return {index};
    if (iequal(type, "ALL")) {
        for (unsigned i = 0; i < L.getnumber(); i++) list[n++] = i;
    } else if (fam.empty()) {
        n = L.findelements(list.data(), type);
        if (index > 0) {
            list[0] = list[index - 1];
            n = 1;
        }
    } else if (!indices.empty()) {
        unsigned nf = L.findelements(list.data(), type, fam, index);
        string idx = indices;
        std::replace(idx.begin(), idx.end(), ',', ' ');
        std::stringstream ss(idx);
        int t;
        n = 0;
        while (ss >> t)
            if (t > 0 && (unsigned)t < nf) list[n++] = list[t - 1];
    } else {
        n = L.findelements(list.data(), type, fam, index);
    }
    list.resize(n);
    return list;
}

// "famname=F1 F2 [a, b] [REPEAT]"
bool two_families(const string& line, string& type, string& f1, string& f2, double& a, double& b,
                  bool& repeat, bool& exact) {
    string u = line;
    size_t lb = u.find('['), rb = u.find(']');
    if (lb == string::npos || rb == string::npos) return false;
    string nums = u.substr(lb + 1, rb - lb - 1);
    std::replace(nums.begin(), nums.end(), ',', ' ');
    std::stringstream(nums) >> a >> b;
    repeat = upper(u.substr(rb)).find("REPEAT") != string::npos;
    exact = upper(u.substr(rb)).find("EXACT") != string::npos;
    string head = u.substr(0, lb);
    size_t pt = upper(head).find("TYPE");
    if (pt != string::npos) {
        size_t e = head.find('=', pt);
        std::stringstream(head.substr(e + 1)) >> type;
        if (!type.empty() && type.back() == ',') type.pop_back();
    }
    size_t pf = upper(head).find("FAMNAME");
    if (pf == string::npos) return false;
    string fams = head.substr(head.find('=', pf) + 1);
    std::replace(fams.begin(), fams.end(), '(', ' ');
    std::replace(fams.begin(), fams.end(), ')', ' ');
    std::replace(fams.begin(), fams.end(), ',', ' ');
    std::stringstream(fams) >> f1 >> f2;
    return !f1.empty() && !f2.empty();
}

struct Deck {
    accel_ctx* ctx = nullptr;
    std::unique_ptr<ALine> L;
    std::vector<double> r;
    int np = 0;
    std::mt19937_64 rng{20171022};
    int mode = ACCEL_MODE_FUSED;

    double gauss() {
        std::normal_distribution<double> g(0.0, 1.0);
        return g(rng);
    }

    void lattice(std::istream& in);
    void optics(std::istream& in);
    void track(std::istream& in);
    void dama(std::istream& in);
    int distribution(const string& line);
};

void Deck::lattice(std::istream& in) {
    const std::vector<string> keys = {"FILE_NAME", "RESET_FIRST", "PRINT_ELEM_VALUE", "PRINT_LAT_SUMMARY",
                                      "EXPORT_ELEMENT", "CORRECT_TUNE", "CORRECT_CHROM", "SET_MAX_NUM_THREADS",
                                      "MODIFY_ELEMENT", "SET_FLAGS", "APPLY_SETPT", "END"};
    string line;
    for (;;) {
        int k = lookfor(in, line, keys);
        if (k < 0 || k == (int)keys.size() - 1) return;
        if (k != 0 && !L) { cout << k << " Lattice file name needs to be given first" << endl; return; }
        auto a = kv(line);
        switch (k) {
        case 0: {
            string rest = line.substr(line.find_first_of("=:") + 1);
            std::replace(rest.begin(), rest.end(), ',', ' ');
            std::stringstream ss(rest);
            string fname, opt;
            ss >> fname;
            int st = 0;
            L.reset(ALine::load(fname, ctx, &st));
            if (!L) { cout << "Exception opening/reading file:" << fname << endl; return; }
            L->mode = mode;
            while (ss >> opt) {
                size_t e = opt.find('=');
                if (e != string::npos && iequal(opt.substr(0, e), "TYPE") && iequal(opt.substr(e + 1), "ERING")) {
                    double phis = L->setrfphase();
                    cout << "RF cavities phase set to: phi_s=" << phis << " rad" << endl;
                    L->set_rad_onoff(0);
                    cout << "radiation off" << endl;
                }
            }
            int ncav = L->set_cavity_onoff(false);
            if (ncav > 0) cout << ncav << " cavity(ies) turned off" << endl;
            int nw = L->set_wake_onoff(false);
            if (nw > 0) cout << nw << " wake element(s) turned off" << endl;
            int ncrab = L->set_crab_onoff(false);
            if (ncrab > 0) cout << ncrab << " crab cavity(ies) turned off" << endl;
            break;
        }
        case 1: {
            // reset_first (process.cpp:280-340): type + famname -> that element; famname alone ->
            // every member of the family in turn, each with its own type and index 1
            string type = get(a, "TYPE"), fam = get(a, "FAMNAME");
            unsigned index = (unsigned)std::atoi(get(a, "INDEX", "1").c_str());
            auto reset = [&](const string& t, unsigned i) {
                cout << "First element moved to: type=" << t << ", famname=" << fam << ", index= " << i << endl;
                unsigned e;
                if (i == 0) std::cerr << "resetfirstelement: element index cannot be zero" << endl;
                if (L->findelements(&e, t, fam, i == 0 ? 1 : i) == 0)
                    cout << "resetfirstelement: element not found (type =" << t << ", famname =" << fam
                         << ", index =" << i << ")" << endl;
                else
                    L->resetfirstelement(e);
            };
            if (!type.empty() && !fam.empty()) {
                reset(type, index);
            } else if (type.empty() && !fam.empty()) {
                unsigned ne = L->getnumber();
                for (unsigned i = 0; i < ne; i++)
                    if (L->element(i).famname == fam) reset(accelgpu::elem_type_name(L->element(i).type), 1);
            }
            break;
        }
        case 2: {
            // print_elem_value: type=T[, famname=F] then the fields to print (process.cpp:343-470);
            // StrMPole knows Index Length PolyB[1..3] PolyA[1..3], Quad knows Index Length K
            string type = get(a, "TYPE"), fam = get(a, "FAMNAME");
            if (type.empty() && fam.empty()) break;
            std::vector<unsigned> list(L->getnumber());
            unsigned n = fam.empty() || type.empty() ? L->findelements(list.data(), type)
                                                     : L->findelements(list.data(), type, fam);
            string rest = line;
            for (const char* key : {"type", "famname"}) {
                std::smatch m;
                if (std::regex_search(rest, m, std::regex(string(key) + R"(\s*=\s*[^\s,]+)", std::regex::icase)))
                    rest = m.prefix().str() + m.suffix().str();
            }
            cout << "$$$Print-Element_Values***********************" << endl;
            for (unsigned i = 0; i < n; i++) {
                const accel_elem_desc& d = L->element(list[i]);
                if (type == "StrMPole") {
                    if (rest.find("Index") != string::npos) cout << list[i] << "\t";
                    if (rest.find("Length") != string::npos) cout << d.len << "\t";
                    for (int j = 1; j <= 3; j++)
                        if (rest.find("PolyB[" + std::to_string(j) + "]") != string::npos) cout << d.poly_b[j] << "\t";
                    for (int j = 1; j <= 3; j++)
                        if (rest.find("PolyA[" + std::to_string(j) + "]") != string::npos) cout << d.poly_a[j] << "\t";
                } else if (type == "Quad") {
                    double kq = 0;
                    L->getfield(list[i], "K", &kq);
                    if (rest.find("Index") != string::npos) cout << list[i] << "\t";
                    if (rest.find("Length") != string::npos) cout << d.len << "\t";
                    if (rest.find("K") != string::npos) cout << kq << "\t";
                }
                cout << endl;
            }
            cout << "******************************************" << endl;
            break;
        }
        case 3: {
            cout << "$$$Lattice-Summary***********************" << endl;
            cout << "Total " << L->getnumber() << " elements, total length = " << L->getlength() << " m" << endl;
            cout << "First element is " << accelgpu::elem_type_name(L->element(0).type) << "." << L->element(0).famname << endl;
            L->set_rad_onoff(0);
            double tx, ty, cx, cy;
            L->calctune(tx, ty);
            cout << "Tunes: " << tx << "\t" << ty << "\t" << endl;
            L->calcchrom(cx, cy);
            cout << "Chromaticity: " << cx << "\t" << cy << "\t" << endl;
            double co[6] = {0, 0, 0, 0, 0, 0};
            L->getco6(co);
            cout << "Closed orbit 6D " << endl;
            for (int i = 0; i < 6; i++) cout << co[i] << "\t";
            cout << endl;
            accelgpu::Twiss tw;
            L->calctwiss(tw);
            cout << "betax\tbetay\talphax\talphay" << endl;
            cout << tw.betx << " \t" << tw.bety << " \t" << tw.alfx << " \t" << tw.alfy << endl;
            cout << "******************************************" << endl;
            break;
        }
        case 4: {
            string type = get(a, "TYPE"), fam = get(a, "FAMNAME");
            // export_element (process.cpp:505-545): RING or LINE writes the whole line with no
            // closing row; a type, or a type and family, writes those elements and a closing row
            bool whole = iequal(type, "RING") || iequal(type, "LINE");
            auto sel = whole ? select(*L, "ALL", "", 0) : select(*L, type, fam, 0);
            cout << "$$$Export-Elements***********************" << endl;
            std::vector<accel_elem_desc> v;
            for (unsigned i : sel) v.push_back(L->element(i));
            ALine tmp(ctx, v);
            tmp.serialize(cout, 6);
            if (!whole) cout << "******************************************" << endl;
            break;
        }
        case 5:
        case 6: {
            // correct_tune / correct_chrom: type=T, famname=(F1 F2) [x, y] [REPEAT] [EXACT]
            // (process.cpp:545-766); EXACT runs Newton iterations on exact one-turn matrices
            const bool tune = (k == 5);
            cout << (tune ? "$$$Correct Tunes***********************" : "$$$Correct chromaticities***********************") << endl;
            string type, f1, f2;
            double t1 = 0, t2 = 0;
            bool repeat = false, exact = false;
            string u = upper(line);
            if (u.find("TYPE") == string::npos || u.find("TYPE") > u.find("FAMNAME")) { cout << "error, specify type first" << endl; break; }
            if (!two_families(line, type, f1, f2, t1, t2, repeat, exact)) { cout << "error, specify famname secondly" << endl; break; }
            cout << type << endl << f1 << " " << f2 << endl;
            cout << (tune ? "Target tunes: " : "Target chromaticities: ") << t1 << "\t" << t2 << "\t" << endl;
            L->set_rad_onoff(0);
            double v1, v2;
            if (tune) {
                L->calctune(v1, v2);
            } else {
                L->set_cavity_onoff(false);
                L->calcchrom(v1, v2);
            }
            cout << (tune ? "Initial tunes: " : "Initial chromaticities: ") << v1 << "\t" << v2 << "\t" << endl;
            std::vector<unsigned> l1(L->getnumber()), l2(L->getnumber());
            unsigned n1 = L->findelements(l1.data(), type, f1), n2 = L->findelements(l2.data(), type, f2);
            if (n1 < 1 || n2 < 1) { cout << "error: no elements found " << n1 << "\t" << n2 << endl; break; }
            cout << n1 << "\t" << n2 << endl;
            for (int p = 0; p < (repeat ? 2 : 1); p++) {
                v1 = t1;
                v2 = t2;
                if (tune && exact) L->correct_tune_exact(v1, v2, n1, n2, l1.data(), l2.data());
                else if (tune) L->correcttune(v1, v2, n1, n2, l1.data(), l2.data());
                else if (exact) L->correct_chrom_exact(v1, v2, n1, n2, l1.data(), l2.data());
                else L->correctchrom(v1, v2, n1, n2, l1.data(), l2.data());
                cout << (tune ? "corrected tunes: " : "corrected chromaticities: ") << v1 << "\t" << v2 << "\t" << endl;
            }
            cout << "*********************************" << endl;
            break;
        }
        case 7: {
            // set_max_num_threads (process.cpp:768-779): the reference's OpenMP thread count.  The
            // tracking here runs on the GPU, so the number is only echoed, with the reference's line.
            string v = line.substr(line.find_first_of("=:") == string::npos ? line.size() : line.find_first_of("=:") + 1);
            int num = 0;
            std::stringstream(v) >> num;
            cout << "Maximum thread number set to " << std::max(num, 1) << endl;
            break;
        }
        case 8: {
            // modify_element: type, famname, index, field, value= | delta= (process.cpp:776-873).
            // As in the reference, `index` both picks the index-th family member (0 = all) and
            // indexes the field's array (PolynomB[index]).
            string type = get(a, "TYPE"), fam = get(a, "FAMNAME"), field = get(a, "FIELD");
            unsigned index = (unsigned)std::atoi(get(a, "INDEX", "0").c_str());
            const bool is_delta = has(a, "DELTA"), is_value = has(a, "VALUE");
            double value = std::atof(get(a, is_delta ? "DELTA" : "VALUE", "0").c_str());
            std::vector<unsigned> list(L->getnumber());
            unsigned n = L->findelements(list.data(), type, fam, index);
            if (n > 0 && (is_delta || is_value)) {
                for (unsigned i = 0; i < n; i++) {
                    double v = value;
                    if (is_delta) {
                        double old = 0;
                        L->getfield(list[i], field, &old, index);
                        v = (field == "NSlice") ? (double)((int)old + (int)value) : old + value;
                    } else if (field == "NSlice") {
                        v = (double)(int)value;
                    }
                    L->setfield(list[i], field, v, index);
                }
            } else {
                if (n == 0) cout << "No element is found: " << type << "\t" << fam << "\t" << index << endl;
                if (!is_delta && !is_value) cout << "No value is given" << endl;
            }
            break;
        }
        case 9: {
            // set_flags (process.cpp:880-965): keys in the order given, each with its message;
            // radiation=lump is this engine's addition and prints nothing
            for (auto& kvp : a) {
                const string& k = kvp.first;
                const string& v = kvp.second;
                int nl = 0;
                if (k == "RADIATION") {
                    if (iequal(v, "OFF")) { L->set_rad_onoff(ACCEL_RAD_OFF); cout << "radiation turned off" << endl; }
                    else if (iequal(v, "RAD") || iequal(v, "ON")) {
                        L->set_rad_onoff(ACCEL_RAD_RAD);
                        cout << "radiation turned on without quantum excitation" << endl;
                    } else if (iequal(v, "RADQE")) {
                        L->set_rad_onoff(ACCEL_RAD_RADQE);
                        cout << "radiation turned on with quantum excitation" << endl;
                    } else if (iequal(v, "LUMP")) L->set_rad_onoff(ACCEL_RAD_LUMP);
                } else if (k == "CAVITY" || k == "CRABCAV" || k == "WAKE") {
                    bool on = iequal(v, "ON");
                    if (!on && !iequal(v, "OFF")) continue;
                    const char* what = k == "CAVITY" ? " cavity(ies) turned " : k == "CRABCAV" ? " crab cavity(ies) turned "
                                                                                                : " wake element(s) turned ";
                    nl = k == "CAVITY" ? L->set_cavity_onoff(on) : k == "CRABCAV" ? L->set_crab_onoff(on) : L->set_wake_onoff(on);
                    if (nl > 0) cout << nl << what << (on ? "on" : "off") << endl;
                }
            }
            break;
        }
        case 10:
            cout << "apply_setpt: not supported by this engine" << endl;
            break;
        }
    }
}

void Deck::optics(std::istream& in) {
    const std::vector<string> keys = {"PRINT_OPTICS", "PRINT_MATRIX", "PRINT_TUNE", "PRINT_CHROM", "PRINT_2ND_CHROM", "END"};
    string line;
    for (;;) {
        int k = lookfor(in, line, keys);
        cout << line << " : " << k << endl;
        if (k < 0 || k == (int)keys.size() - 1) return;
        if (!L) return;
        auto a = kv(line);
        double dpp = std::atof(get(a, "DPP", "0").c_str());
        double delta = std::atof(get(a, "DELTA", "1e-8").c_str());
        string idx = get(a, "INDEX", "0"), indices;
        if (!idx.empty() && idx[0] == '[') { indices = idx.substr(1, idx.size() - 2); idx = "0"; }
        string type = get(a, "TYPE"), fam = get(a, "FAMNAME");
        if (k == 0) {
            auto sel = select(*L, type, fam, (unsigned)std::atoi(idx.c_str()), indices);
            std::vector<accelgpu::Twiss> tw(sel.size());
            cout << "nlist=" << sel.size() << endl;
            if (!sel.empty()) L->calctwiss(tw.data(), sel.data(), (int)sel.size(), dpp, delta);
            cout << "$$$Optics-Twiss, dp=" << dpp << "*************************** " << sel.size() << " points" << endl;
            cout << "index\ts (m)\tbetx (m)\tbety (m)\talfx\talfy\tpsix\tpsiy\n";
            for (size_t i = 0; i < sel.size(); i++)
                cout << sel[i] << "\t" << tw[i].s << "\t" << tw[i].betx << "\t" << tw[i].bety << "\t" << tw[i].alfx << "\t"
                     << tw[i].alfy << "\t" << tw[i].psix << "\t" << tw[i].psiy << "\t" << endl;
        } else if (k == 1) {
            string style = get(a, "LINE_STYLE", "6by6");
            auto print = [&](const double* m) {
                int n = iequal(style, "4by4") ? 4 : 6;
                if (iequal(style, "oneline")) {
                    for (int i = 0; i < 36; i++) cout << m[i] << "\t";
                    cout << endl;
                } else if (iequal(style, "4by4") || iequal(style, "6by6")) {
                    for (int i = 0; i < n; i++) {
                        for (int j = 0; j < n; j++) cout << m[6 * i + j] << "\t";
                        cout << endl;
                    }
                }
            };
            double m[36];
            if (iequal(type, "RING") || iequal(type, "ONETURN")) {
                L->getm66(m, dpp, delta);
                cout << "$$$OPTICS-MATRIX*******************ONE-TURN" << endl;
                cout << "type=RING at " << accelgpu::elem_type_name(L->element(0).type) << ", famname=" << L->element(0).famname
                     << ", ring index=" << 0 << ", spos=" << L->getlength() << endl;
                print(m);
                cout << "****************************" << endl;
            } else {
                auto sel = select(*L, type, fam, (unsigned)std::atoi(idx.c_str()), indices);
                if (!sel.empty()) cout << "$$$OPTICS-MATRIX, dpp=" << dpp << "******************* " << sel.size() << " points" << endl;
                else cout << "#no element found for matrix print out, type=" << type << ", famname=" << fam << ",index" << idx << endl;
                for (unsigned e : sel) {
                    L->getm66(m, 0, e, dpp, delta);
                    cout << "type=" << type << ", famname=" << fam << ", ring index=" << e << ", spos=" << L->getlength(e) << endl;
                    print(m);
                }
                if (!sel.empty()) cout << "**********************" << endl;
            }
        } else {
            L->set_rad_onoff(0);
            double x, y;
            if (k == 2) {
                L->calctune(x, y, dpp, delta);
                cout << "Tunes: [" << x << "\t" << y << "], dpp=" << dpp << endl;
            } else if (k == 3) {
                L->calcchrom(x, y, dpp, delta);
                cout << "Chromaticity: [" << x << "\t" << y << "], dpp=" << dpp << endl;
            } else {
                double x2, y2;
                L->calcchrom2(x, y, x2, y2);
                cout << "Chromaticity: [" << x << "\t" << y << "]" << endl;
                cout << "2nd-order Chromaticity: [" << x2 << "\t" << y2 << "], " << endl;
            }
        }
    }
}

int Deck::distribution(const string& line_in) {
    cout << line_in << endl;
    string line = line_in;
    string sel = line.substr(line.find_first_of("=:") + 1);
    trim(sel);
    r.clear();
    if (sel.empty()) { r.assign(6, 0.0); return 1; }
    std::stringstream ss(sel);
    string opt;
    ss >> opt;
    auto a = kv(": " + sel.substr(opt.size()));
    auto num = [&](const string& k, double d) { return has(a, k) ? std::atof(get(a, k).c_str()) : d; };
    if (iequal(opt, "ZERO")) {
        int n = (int)num("NPAR", 1);
        r.assign((size_t)6 * std::max(0, n), 0.0);
        return std::max(0, n);
    }
    if (iequal(opt, "COORDINATE")) {
        size_t b = sel.find('('), e = sel.find(')');
        string body = sel.substr(b + 1, e - b - 1);
        std::replace(body.begin(), body.end(), ',', ' ');
        std::stringstream bs(body);
        string part;
        while (std::getline(bs, part, ';')) {
            std::stringstream ps(part);
            double v[6] = {0, 0, 0, 0, 0, 0};
            for (int j = 0; j < 6; j++) ps >> v[j];
            r.insert(r.end(), v, v + 6);
        }
        return (int)(r.size() / 6);
    }
    if (iequal(opt, "GAUSSIAN")) {
        int n = (int)num("NPAR", 1);
        double sigx = num("SIGX", 0), sigxp = num("SIGXP", 0), sigy = num("SIGY", 0), sigyp = num("SIGYP", 0);
        if (has(a, "EMIT_X") || has(a, "EMIT_Y")) {
            accelgpu::Twiss tw;
            L->calctwiss(tw);
            double bx = num("BETX", std::isnan(tw.betx) ? 1.0 : tw.betx);
            double by = num("BETY", std::isnan(tw.bety) ? 1.0 : tw.bety);
            if (has(a, "EMIT_X")) { sigx = std::sqrt(bx * num("EMIT_X", 0)); sigxp = std::sqrt(num("EMIT_X", 0) / bx); }
            if (has(a, "EMIT_Y")) { sigy = std::sqrt(by * num("EMIT_Y", 0)); sigyp = std::sqrt(num("EMIT_Y", 0) / by); }
        }
        double sigz = num("SIGZ", 0), sigd = num("SIGDPP", num("SIGDP", 0));
        r.resize((size_t)6 * n);
        for (int i = 0; i < n; i++) {
            double* p = &r[(size_t)6 * i];
            p[0] = gauss() * sigx; p[1] = gauss() * sigxp; p[2] = gauss() * sigy;
            p[3] = gauss() * sigyp; p[4] = gauss() * sigz; p[5] = gauss() * sigd;
        }
        return n;
    }
    if (iequal(opt, "LINEAR")) {
        // Linear C=start:step:end (process.cpp:1761-1802): the first key names the swept
        // coordinate (X XP Y YP Z DELTA; anything else sweeps X), the others stay zero; the count
        // comes from stepping a running value, the values are start + step * i
        const char* names[6] = {"X", "XP", "Y", "YP", "Z", "DELTA"};
        string key, spec;
        for (auto& kvp : a)
            if (!kvp.second.empty()) { key = kvp.first; spec = kvp.second; break; }
        int c = 0;
        for (int j = 0; j < 6; j++)
            if (key == names[j]) c = j;
        if (key == "DP") c = 5;
        std::replace(spec.begin(), spec.end(), ':', ' ');
        double lo = 0, st = 0, hi = 0;
        std::stringstream(spec) >> lo >> st >> hi;
        if (st == 0) { cout << "interval cannot be zero" << endl; return 0; }
        int n = 0;
        for (double v = lo; (v <= hi && st > 0) || (v >= hi && st < 0); v += st) n++;
        r.assign((size_t)6 * n, 0.0);
        for (int i = 0; i < n; i++) r[(size_t)6 * i + c] = lo + st * i;
        return n;
    }
    if (iequal(opt, "LOAD")) {
        // Load FILE[, format=plain|accel-export] (process.cpp:1471-1555): the file name is echoed;
        // an accel-export file is read from its "Full export" block, whose Np line and data lines
        // are echoed as they are read; lines of 11 characters or fewer and "%" lines are skipped
        string fname;
        ss >> fname;
        if (!fname.empty() && fname.back() == ',') fname.pop_back();
        cout << fname << endl;
        if (upper(sel).find("FORMAT=BINARY") != string::npos) {
            // this engine's lossless checkpoint (Do_Track save=FILE, accel_state_write)
            double* rr = nullptr;
            int64_t n = 0, t = 0;
            int st = accel_state_read(fname.c_str(), &rr, &n, &t, nullptr);
            if (st) { cout << "cannot load " << fname << ": " << accel_last_error() << endl; return 0; }
            r.assign(rr, rr + 6 * n);
            accel_state_free(rr);
            return (int)n;
        }
        bool exported = upper(sel).find("ACCEL-EXPORT") != string::npos;
        std::ifstream f(fname);
        string sl;
        if (exported)
            while (mgetline(f, sl))
                if (sl.compare(0, 3, "$$$") == 0 && sl.find("Full export") != string::npos) {
                    mgetline(f, sl);
                    cout << sl << endl;
                    break;
                }
        while (mgetline(f, sl)) {
            if (sl.compare(0, 5, "*****") == 0) break;
            trim(sl);
            if (sl.size() <= 11 || sl[0] == '%') continue;
            if (exported) cout << sl << endl;
            std::stringstream ls(sl);
            double t, v[6] = {0, 0, 0, 0, 0, 0};
            if (exported) ls >> t;
            for (int j = 0; j < 6; j++) ls >> v[j];
            r.insert(r.end(), v, v + 6);
        }
        return (int)(r.size() / 6);
    }
    cout << "unknown distribution option " << opt << endl;
    return 0;
}

void Deck::track(std::istream& in) {
    const std::vector<string> keys = {"DISTRIBUTION", "MONITOR", "DO_TRACK", "TRANSPORT", "END"};
    string line;
    for (;;) {
        int k = lookfor(in, line, keys);
        if (k < 0 || k == (int)keys.size() - 1) return;
        if (!L) return;
        auto a = kv(line);
        if (k == 0) {
            np = distribution(line);
            string u = upper(line);
            size_t ps = u.find("SHIFT");
            if (np > 0 && ps != string::npos) {
                size_t b = u.find('(', ps), e = u.find(')', b);
                string s = line.substr(b + 1, e - b - 1);
                std::replace(s.begin(), s.end(), ',', ' ');
                double d[6] = {0, 0, 0, 0, 0, 0};
                std::stringstream(s) >> d[0] >> d[1] >> d[2] >> d[3] >> d[4] >> d[5];
                for (int i = 0; i < np; i++)
                    for (int j = 0; j < 6; j++) r[(size_t)6 * i + j] += d[j];
            }
            if (u.find("PRINT") != string::npos) {
                cout << "$$$Init-Distribution*************" << endl;
                for (int i = 0; i < np; i++) {
                    for (int j = 0; j < 6; j++) cout << r[(size_t)6 * i + j] << " ";
                    cout << endl;
                }
                cout << "***********************" << endl;
            }
        } else if (k == 1) {
            accel_elem_desc m;
            accel_elem_default(ACCEL_MONITOR, &m);
            std::snprintf(m.famname, sizeof(m.famname), "FirstMonitor");
            int interval = std::max(1, std::atoi(get(a, "INTERVAL", "1").c_str()));
            double frac = std::min(1.0, std::max(0.01, std::atof(get(a, "FRACTION", "1.0").c_str())));
            m.f[0] = interval;
            m.f[1] = frac;
            L->insertelement(0, m);
            string fl = get(a, "PRINTFLAG", "COORDINATE");
            if (iequal(fl, "COORDINATE")) L->set_monitor(accelgpu::MON_COORD, 1);
            else if (iequal(fl, "STAT1")) L->set_monitor(accelgpu::MON_STAT1, 1);
            else if (iequal(fl, "STAT2")) L->set_monitor(accelgpu::MON_STAT2, 1);
        } else if (k == 2) {
            string rad = get(a, "RADIATION"), rf = get(a, "RFCAVITY"), pf = get(a, "PRINTFINAL", "NO");
            int nturn = std::atoi(get(a, "NTURN", "0").c_str());
            if (iequal(rad, "OFF")) L->set_rad_onoff(ACCEL_RAD_OFF);
            else if (iequal(rad, "RAD")) L->set_rad_onoff(ACCEL_RAD_RAD);
            else if (iequal(rad, "RADQE")) L->set_rad_onoff(ACCEL_RAD_RADQE);
            else if (iequal(rad, "LUMP")) L->set_rad_onoff(ACCEL_RAD_LUMP);
            else if (iequal(rad, "LUMPDAMP")) L->set_rad_onoff(ACCEL_RAD_LUMP_DAMP);
            else if (iequal(rad, "LUMPQE")) L->set_rad_onoff(ACCEL_RAD_LUMP_QE);
            if (iequal(rf, "OFF")) L->set_cavity_onoff(false);
            else if (iequal(rf, "ON")) L->set_cavity_onoff(true);
            if (np > 0 && nturn > 0) {
                // the reference reads "PrintFlag" from element 0 whatever its type
                // (process.cpp:2000-2002); the multipole classes report the missing field
                // (accel.cpp:619, 770) and the flag is then unset there; here nothing is printed
                int t0 = L->element(0).type;
                if (t0 == ACCEL_STRMPOLE || t0 == ACCEL_BENDMPOLE)
                    cout << (t0 == ACCEL_STRMPOLE ? "AStrMPole" : "ABendMPole")
                         << "::getfield() --> no matched field PrintFlag" << endl;
                unsigned flag = L->monitor_flag();
                if (flag == accelgpu::MON_COORD) {
                    double ratio = L->element(0).type == ACCEL_MONITOR ? L->element(0).f[1] : 1.0;
                    int iskip = std::min(np, std::max(1, (int)(1. / ratio)));
                    cout << "$$$Track-Data: Coordinate**************************" << endl;
                    cout << "#" << rad << " " << rf << " " << nturn << endl;
                    cout << "Np=" << np << ", Nprint=" << np / iskip << endl;
                } else if (flag == accelgpu::MON_STAT1 || flag == accelgpu::MON_STAT2) {
                    cout << (flag == accelgpu::MON_STAT1 ? "$$$Track-Data: Stat1" : "$$$Track-Data: Stat2")
                         << "******************************" << endl;
                    cout << "#" << rad << " " << rf << " " << nturn << endl;
                    cout << "Np=" << np << endl;
                }
                L->set_monitor_pass(0);
                int st = L->pass(r.data(), np, nturn);
                if (st) cout << "tracking failed: " << accel_status_string(st) << " " << accel_last_error() << endl;
                if (iequal(pf, "Full")) {
                    cout << "*************************************" << endl;
                    cout << "$$$Track-Data: Full export ************************" << endl;
                    cout << "Np=" << np << ", Nprint=" << np << endl;
                    for (int i = 0; i < np; i++) {
                        cout << nturn << "\t";
                        for (int j = 0; j < 6; j++) cout << r[(size_t)6 * i + j] << "\t";
                        cout << endl;
                    }
                } else if (iequal(pf, "Yes") || iequal(pf, "same")) {
                    L->monitor_print(r.data(), np, nturn, cout);
                }
                // save=FILE (an extension): the final distribution as a lossless checkpoint, read
                // back by "Distribution : Load FILE, format=binary"
                const string save = get(a, "SAVE");
                if (!save.empty() && accel_state_write(save.c_str(), r.data(), np, nturn, nullptr))
                    cout << "cannot save " << save << ": " << accel_last_error() << endl;
                cout << "*************************************" << endl;
            }
        } else if (k == 3) {
            // Transport (process.cpp:2108-2205): index=N or an index list index=[i, j, ...].  At
            // each watch point the reference prints the block's distribution as the last Do_Track
            // left it; its transported copy is advanced but not printed.  This deck does the same.
            string type = get(a, "TYPE"), fam = get(a, "FAMNAME"), idx = get(a, "INDEX", "0"), indices;
            unsigned index = 0;
            if (!idx.empty() && idx[0] == '[') {
                indices = idx.substr(1, idx.size() - 2);
                std::replace(indices.begin(), indices.end(), ',', ' ');
                size_t b = indices.find_first_not_of(" \t"), e = indices.find_last_not_of(" \t");
                indices = (b == string::npos) ? string() : indices.substr(b, e - b + 1);
                indices += " ";
            } else {
                index = (unsigned)std::atoi(idx.c_str());
            }
            auto sel = select(*L, type, fam, index, indices);
            cout << type << " " << fam << " ";
            if (indices.empty()) cout << index << endl;
            else cout << indices << endl;
            if (sel.empty()) { cout << "No watch point found" << endl; continue; }
            std::vector<double> nr = r;
            cout << "$$$Track-Transport: ************************" << endl;
            unsigned prev = 0;
            for (unsigned e : sel) {
                L->pass(nr.data(), np, prev, e);
                cout << "type=" << type << ", famname=" << fam << ", ring index=" << e << ", spos=" << L->getlength(e) << endl;
                for (int i = 0; i < np; i++) {
                    cout << e << "\t";
                    for (int j = 0; j < 6; j++) cout << r[(size_t)6 * i + j] << "\t";
                    cout << endl;
                }
                cout << "#------end of ring index=" << e << endl;
                prev = e;
            }
            cout << "******************************" << endl;
        }
    }
}

void Deck::dama(std::istream& in) {
    const std::vector<string> keys = {"APPLY_SETPT", "TRACK_DA", "TRACK_MA", "TRACK_DNUDJ", "END"};
    string line;
    for (;;) {
        int k = lookfor(in, line, keys);
        if (k < 0 || k == (int)keys.size() - 1) return;
        if (!L) return;
        auto a = kv(line);
        if (k == 1) {
            double xmin = std::atof(get(a, "XMIN").c_str()), xmax = std::atof(get(a, "XMAX").c_str());
            double ymax = std::atof(get(a, "YMAX").c_str());
            int nray = std::atoi(get(a, "NRAY").c_str()), nstep = std::atoi(get(a, "NSTEP").c_str());
            int nturn = std::atoi(get(a, "NTURN").c_str());
            bool neg = iequal(get(a, "WEIGHTMINUSSIDE"), "true");
            double rx[51], ry[51];
            if (nray < 2 || nray > 51) cout << "Error: number of rays: " << nray << endl;
            L->set_monitor(0, 1);
            cout << "#" << xmin << " " << xmax << " " << ymax << " " << nray << " " << nstep << " " << nturn << " " << neg << endl;
            L->set_rad_onoff(ACCEL_RAD_RAD);
            L->set_cavity_onoff(true);
            cout << "#" << now() << endl;
            double S = L->trackDA(xmax, xmin, ymax, nturn, (unsigned)nray, nstep, rx, ry, neg);
            cout << "$$$DA-profile " << nturn << " turns, " << (neg ? "3/4 DA area=" : "DA area=") << S * 1.0e6 << " mm^2" << endl;
            for (int i = 0; i < std::min(51, std::max(3, nray)); i++) cout << rx[i] << " \t" << ry[i] << " \t" << endl;
            cout << "#" << now() << endl;
            cout << "******************************" << endl;
        } else if (k == 2) {
            string type = get(a, "TYPE"), fam = get(a, "FAMNAME");
            auto sel = select(*L, type, fam, 0);
            unsigned nmoni = (unsigned)std::atoi(get(a, "NMONI", "0").c_str());
            int nstep = std::atoi(get(a, "NSTEP").c_str()), nturn = std::atoi(get(a, "NTURN").c_str());
            double dmin = std::atof(get(a, "DPPMIN").c_str()), dmax = std::atof(get(a, "DPPMAX").c_str());
            cout << "#" << nmoni << " " << nstep << " " << nturn << " " << dmin << " " << dmax << endl;
            if (nmoni > sel.size()) nmoni = (unsigned)sel.size();
            std::vector<double> dp(nmoni), dm(nmoni);
            L->set_rad_onoff(ACCEL_RAD_RAD);
            L->set_cavity_onoff(true);
            cout << "#" << now() << endl;
            double avg = L->trackMA(dmax, dmin, nturn, (unsigned)nstep, dp.data(), dm.data(), nmoni, sel.data());
            cout << "$$$MA " << nturn << " turns, average MA=" << avg << endl;
            for (unsigned i = 0; i < nmoni; i++) cout << dp[i] << " \t" << dm[i] << " \t" << endl;
            cout << "#" << now() << endl;
            cout << "******************************" << endl;
        } else if (k == 3) {
            // track_dNudJ: amplitude-dependent tune shift (process.cpp:2590-2628)
            double xm = std::atof(get(a, "XMAX").c_str()), ym = std::atof(get(a, "YMAX").c_str());
            unsigned nturn = (unsigned)std::atoi(get(a, "NTURN").c_str());
            cout << "#" << xm << " " << ym << " " << nturn << endl;
            double d[4];
            L->set_monitor(0, 0);
            L->set_rad_onoff(0);
            L->set_cavity_onoff(false);
            L->trackdnudexy(d, nturn, xm, ym, &cout);
            cout << "$$$dtuning coefficients" << endl;
            cout << d[0] << " \t" << d[1] << " \t" << d[2] << " \t" << d[3] << " \t" << endl;
            cout << "*************************" << endl;
        } else {
            cout << "apply_setpt: not supported by this engine" << endl;
        }
    }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "usage: accel+gpu DECK [--device N] [--plain | --exact] [--seed S]" << std::endl;
        return 1;
    }
    Deck D;
    int device = 0;
    for (int i = 2; i < argc; i++) {
        if (!std::strcmp(argv[i], "--device") && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--plain")) D.mode = ACCEL_MODE_PLAIN;
        else if (!std::strcmp(argv[i], "--exact")) D.mode = ACCEL_MODE_EXACT;
        else if (!std::strcmp(argv[i], "--seed") && i + 1 < argc) D.rng.seed(std::strtoull(argv[++i], nullptr, 10));
    }
    std::ifstream fin(argv[1]);
    if (!fin.good()) { std::cerr << "cannot open " << argv[1] << std::endl; return 1; }
    int s = accel_ctx_create(device, &D.ctx);
    if (s) {
        std::cerr << "accel+gpu: " << accel_status_string(s) << ": " << accel_last_error() << std::endl;
        return 2;
    }
    const std::vector<string> blocks = {"LATTICE", "OPTICS", "SURVEY", "DAMA", "TRACK"};
    string line;
    int b = lookfor(fin, line, blocks);
    if (b > 0) { cout << "The first block must be LATTICE." << endl; return 1; }
    if (b < 0) { cout << "No LATTICE block is found." << endl; return 1; }
    cout << "#" << now() << endl;
    D.lattice(fin);
    if (!D.L) { accel_ctx_destroy(D.ctx); return 1; }
    cout << "Total elements: " << D.L->getnumber() << endl;
    for (;;) {
        int k = lookfor(fin, line, blocks);
        if (k < 0) break;
        cout << blocks[k] << endl;
        if (k == 0) D.lattice(fin);
        else if (k == 1) D.optics(fin);
        else if (k == 3) D.dama(fin);
        else if (k == 4) {
            cout << "#" << now() << endl;
            D.track(fin);
            cout << "#" << now() << endl;
        }
    }
    D.L.reset();
    accel_ctx_destroy(D.ctx);
    return 0;
}
