// host_aline.cpp — ALine over the GPU C-ABI (see host_aline.hpp).
#include "host_aline.hpp"

#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>
#include "engine.h"
#include "runtime.h"

namespace accelgpu {

namespace {
const double kPi = 3.1415926535897932384626;

int field_id(const std::string& name) {
    static const struct { const char* n; int id; } T[] = {
        {"Length", ACCEL_F_LENGTH}, {"K", ACCEL_F_K}, {"PolynomB", ACCEL_F_POLYNOMB},
        {"PolynomA", ACCEL_F_POLYNOMA}, {"NSlice", ACCEL_F_NSLICE}, {"MaxNPole", ACCEL_F_MAXNPOLE},
        {"BendingAngle", ACCEL_F_ANGLE}, {"EntranceAngle", ACCEL_F_E1}, {"ExitAngle", ACCEL_F_E2},
        {"Voltage", ACCEL_F_VOLTAGE}, {"Frequency", ACCEL_F_FREQUENCY}, {"Phis", ACCEL_F_PHIS},
        {"Energy", ACCEL_F_ENERGY}, {"energy", ACCEL_F_ENERGY}, {"KickX", ACCEL_F_KICKX},
        {"KickY", ACCEL_F_KICKY}, {"XLim", ACCEL_F_XLIM}, {"YLim", ACCEL_F_YLIM}};
    for (auto& t : T)
        if (name == t.n) return t.id;
    return 0;
}

// Solve (I - M) x = b for an n x n block of a 6x6 row-major M (Gaussian elimination with
// partial pivoting).  The reference inverts through an SVD (MatVec); any exact solve agrees.
bool solve_I_minus(const double* m66, int n, const double* b, double* x) {
    double a[6][7];
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++) a[i][j] = (i == j ? 1.0 : 0.0) - m66[6 * i + j];
        a[i][n] = b[i];
    }
    for (int c = 0; c < n; c++) {
        int p = c;
        for (int r = c + 1; r < n; r++)
            if (std::fabs(a[r][c]) > std::fabs(a[p][c])) p = r;
        if (a[p][c] == 0.0) return false;
        if (p != c)
            for (int k = 0; k <= n; k++) std::swap(a[p][k], a[c][k]);
        for (int r = 0; r < n; r++) {
            if (r == c) continue;
            double f = a[r][c] / a[c][c];
            for (int k = c; k <= n; k++) a[r][k] -= f * a[c][k];
        }
    }
    for (int i = 0; i < n; i++) x[i] = a[i][n] / a[i][i];
    return true;
}
}  // namespace

double tune_of(const double* m, int k) { return std::acos((m[6 * k + k] + m[6 * (k + 1) + k + 1]) * 0.5) / 2.0 / kPi; }

const char* elem_type_name(int type) { return accel::type_name(type); }

// ---- NAFF ----------------------------------------------------------------------------------------
namespace {
// -|windowed projection| at frequency nu (the quantity the search minimises)
double projection(double nu, int N, const double* X) {
    double re = 0, im = 0;
    for (int i = 0; i < N; i++) {
        const double ph = 2 * kPi * nu * i;
        const double w = std::pow(std::sin(kPi * i / N), 4);
        re += std::cos(ph) * X[i] * w;
        im -= std::sin(ph) * X[i] * w;
    }
    return -std::sqrt(re * re + im * im);
}

// power of the packed real spectrum at even index i: (F_0^2 + F_{N/2}^2) at 0, |F_{i/2}|^2 else
double packed_power(int N, const double* X, int i) {
    auto dft = [&](int k, double& re, double& im) {
        re = im = 0;
        for (int j = 0; j < N; j++) {
            const double ph = 2 * kPi * (double)k * j / N;
            re += X[j] * std::cos(ph);
            im += X[j] * std::sin(ph);
        }
    };
    double r0, i0, r1, i1;
    if (i == 0) {
        dft(0, r0, i0);
        dft(N / 2, r1, i1);
        return r0 * r0 + r1 * r1;
    }
    dft(i / 2, r0, i0);
    return r0 * r0 + i0 * i0;
}

// golden-section search for a minimum of f on [a, c] with interior guess b
template <class F>
double golden_min(F f, double a, double b, double c, double tol) {
    const double R = 0.61803398874989484820, C = 1 - R;
    double x0 = a, x3 = c, x1, x2;
    if (std::fabs(c - b) > std::fabs(b - a)) { x1 = b; x2 = b + C * (c - b); }
    else { x2 = b; x1 = b - C * (b - a); }
    double f1 = f(x1), f2 = f(x2);
    while (std::fabs(x3 - x0) > tol * (std::fabs(x1) + std::fabs(x2))) {
        if (f2 < f1) {
            x0 = x1; x1 = x2; x2 = R * x2 + C * x3;
            f1 = f2; f2 = f(x2);
        } else {
            x3 = x2; x2 = x1; x1 = R * x1 + C * x0;
            f2 = f1; f1 = f(x1);
        }
    }
    return f1 < f2 ? x1 : x2;
}

void fit_slope(int n, const double* x, const double* y, double& slope) {
    double sx = 0, sy = 0;
    for (int i = 0; i < n; i++) { sx += x[i]; sy += y[i]; }
    const double mx = sx / n, my = sy / n;
    double sxx = 0, sxy = 0;
    for (int i = 0; i < n; i++) { sxx += (x[i] - mx) * (x[i] - mx); sxy += (x[i] - mx) * (y[i] - my); }
    slope = sxy / sxx;
}

unsigned pow2_at_least(unsigned n) {
    unsigned nt = 1;
    while (nt < n) nt <<= 1;
    return nt;
}
}  // namespace

double naff(int N, const double* X, double xlow, double xhi) {
    xlow = std::max(xlow, 0.9 / N);
    xhi = std::min(0.5, xhi);
    const int ilow = ((int)(xlow * N * 2) >> 1) << 1;
    const int ihi = ((int)(xhi * N * 2) >> 1) << 1;
    int im = ilow;
    double fm = packed_power(N, X, ilow);
    for (int i = ilow + 2; i < ihi; i += 2) {
        const double f = packed_power(N, X, i);
        if (f > fm) { im = i; fm = f; }
    }
    xlow = std::max(xlow, (im - 2) * 1.0 / N / 2.0);
    xhi = std::min(xhi, (im + 2) * 1.0 / N / 2.0);
    return golden_min([&](double nu) { return projection(nu, N, X); }, xlow, 0.5 * (xlow + xhi), xhi, 3.0e-8);
}

void Twiss::serialize(std::ostream& os) const {
    os << s << "\t" << betx << "\t" << bety << "\t" << alfx << "\t" << alfy << "\t" << psix << "\t" << psiy << "\t" << std::endl;
}

ALine::ALine(accel_ctx* ctx, std::vector<accel_elem_desc> elems) : ctx_(ctx), desc_(std::move(elems)) {}

ALine::~ALine() {
    if (line_) accel_line_destroy(line_);
}

ALine* ALine::deserialize(std::istream& is, accel_ctx* ctx, int* status) {
    std::stringstream ss;
    ss << is.rdbuf();
    accel_elem_desc* e = nullptr;
    int n = 0;
    int s = accel_lattice_parse(ss.str().c_str(), &e, &n);
    if (status) *status = s;
    if (s) return nullptr;
    std::vector<accel_elem_desc> v(e, e + n);
    accel_lattice_free(e);
    return new ALine(ctx, std::move(v));
}

ALine* ALine::load(const std::string& path, accel_ctx* ctx, int* status) {
    std::ifstream f(path);
    if (!f.good()) {
        if (status) *status = ACCEL_E_IO;
        return nullptr;
    }
    return deserialize(f, ctx, status);
}

int ALine::sync() {
    if (!dirty_ && line_) return ACCEL_OK;
    if (line_) { accel_line_destroy(line_); line_ = nullptr; }
    status_ = accel_line_create(ctx_, desc_.data(), (int)desc_.size(), &line_);
    if (status_ == ACCEL_OK) dirty_ = false;
    return status_;
}

accel_line* ALine::device_line() { return sync() == ACCEL_OK ? line_ : nullptr; }

double ALine::getlength(unsigned st, unsigned ed) const {
    double len = 0.;
    for (unsigned i = st; i < ed && i < desc_.size(); i++) len += desc_[i].len;
    return len;
}

int ALine::addelement(const accel_elem_desc& e) { desc_.push_back(e); dirty_ = true; return (int)desc_.size(); }
int ALine::insertelement(unsigned i, const accel_elem_desc& e) {
    if (i > desc_.size()) return (int)desc_.size();
    desc_.insert(desc_.begin() + i, e);
    dirty_ = true;
    return (int)desc_.size();
}
int ALine::deleteelement(unsigned i) {
    if (i < desc_.size()) { desc_.erase(desc_.begin() + i); dirty_ = true; }
    return (int)desc_.size();
}

unsigned ALine::findelements(unsigned* list, const std::string& type, const std::string& famname,
                             unsigned index) const {
    unsigned cnt = 0;
    for (unsigned i = 0; i < desc_.size(); i++) {
        if (accel::type_name(desc_[i].type) == type && famname == desc_[i].famname) {
            cnt++;
            if (index == 0) list[cnt - 1] = i;
            else if (index == cnt) { list[0] = i; return 1; }
        }
    }
    return index == 0 ? cnt : 0;
}

unsigned ALine::findelements(unsigned* list, const std::string& type) const {
    unsigned cnt = 0;
    for (unsigned i = 0; i < desc_.size(); i++)
        if (accel::type_name(desc_[i].type) == type) list[cnt++] = i;
    return cnt;
}

unsigned ALine::resetfirstelement(unsigned eindex) {
    if (eindex == 0 || eindex >= desc_.size()) return 0;
    std::rotate(desc_.begin(), desc_.begin() + eindex, desc_.end());
    dirty_ = true;
    return (unsigned)desc_.size() - eindex;
}

unsigned ALine::resetfirstelement(const std::string& type, const std::string& famname, unsigned index) {
    unsigned e;
    if (findelements(&e, type, famname, index == 0 ? 1 : index) == 0) return 0;
    return resetfirstelement(e);
}

void ALine::serialize(std::ostream& os, int precision) const {
    os << accel::format_lattice(desc_.data(), (int)desc_.size(), precision);
}

int ALine::setenergy(double en) {
    int cnt = 0;
    for (auto& d : desc_)
        if (d.type == ACCEL_CAVITY || d.type == ACCEL_BENDMPOLE || d.type == ACCEL_TRANSWAKE ||
            d.type == ACCEL_LONGWAKE || d.type == ACCEL_CRABCAV || d.type == ACCEL_RFMULT ||
            d.type == ACCEL_IDEALWIG) {
            double v = en;
            accel::desc_set_field(d, ACCEL_F_ENERGY, 0, &v);
            if (d.type == ACCEL_CRABCAV) d.f[4] = en;
            if (d.type == ACCEL_RFMULT) d.f[2] = en;
            cnt++;
        }
    dirty_ = true;
    return cnt;
}

int ALine::set_rad_onoff(unsigned flag) {
    int cnt = 0;
    for (auto& d : desc_)
        if (d.type == ACCEL_BENDMPOLE || d.type == ACCEL_IDEALWIG || d.type == ACCEL_SYNCRAD) cnt++;
    accel::apply_flags(desc_.data(), (int)desc_.size(), (int)flag, -1, -1);
    dirty_ = true;
    return cnt;
}

int ALine::set_cavity_onoff(bool flag) {
    int cnt = 0;
    for (auto& d : desc_)
        if (d.type == ACCEL_CAVITY) { d.flags = flag ? 1 : 0; cnt++; }
    dirty_ = true;
    return cnt;
}

int ALine::set_crab_onoff(bool flag) {  // aline.cpp:441-450
    int n = 0;
    for (auto& d : desc_)
        if (d.type == ACCEL_CRABCAV) { d.flags = flag ? 1 : 0; n++; }
    dirty_ = true;
    return n;
}

int ALine::set_wake_onoff(bool flag) {
    int cnt = 0;
    for (auto& d : desc_)
        if (d.type == ACCEL_TRANSWAKE || d.type == ACCEL_LONGWAKE) { d.flags = flag ? 1 : 0; cnt++; }
    dirty_ = true;
    return cnt;
}

int ALine::set_monitor(unsigned flag, unsigned index) {
    // the monitor that prints is the one at element 0 (the Track block inserts it there)
    unsigned cnt = 0;
    for (unsigned i = 0; i < desc_.size(); i++)
        if (desc_[i].type == ACCEL_MONITOR) {
            cnt++;
            if ((index == 0 || index == cnt) && i == 0) mon_flag_ = flag;
            if (index == cnt) break;
        }
    return 0;
}

int ALine::set_monitor_pass(int num) { mon_cnt_pass_ = num; return 1; }

double ALine::setrfphase() {
    if (sync()) return 0;
    double phis = 0;
    status_ = accel_line_setrfphase(line_, &phis);
    if (status_) return 0;
    // copy the phase and the switches (cavities off, radiation off) back to the host copy
    for (unsigned i = 0; i < desc_.size(); i++) accel_line_get_desc(line_, (int)i, &desc_[i]);
    dirty_ = true;
    return phis;
}

double ALine::setrfphase(double phis) {
    for (auto& d : desc_)
        if (d.type == ACCEL_CAVITY) d.f[2] = phis;
    dirty_ = true;
    return phis;
}

int ALine::setfield(unsigned idx, const std::string& name, double value, unsigned index) {
    if (idx >= desc_.size()) return ACCEL_E_INVALID;
    int id = field_id(name);
    if (!id) return ACCEL_E_INVALID;
    double v[2] = {value, value};
    int s = accel::desc_set_field(desc_[idx], id, (int)index, v);
    if (!s) dirty_ = true;
    return s;
}

int ALine::getfield(unsigned idx, const std::string& name, double* value, unsigned index) const {
    if (idx >= desc_.size()) return ACCEL_E_INVALID;
    int id = field_id(name);
    if (!id) return ACCEL_E_INVALID;
    return accel::desc_get_field(desc_[idx], id, (int)index, value);
}

// ---- tracking ------------------------------------------------------------------------------------
int ALine::pass(double* r, int N, unsigned st, unsigned ed) {
    if ((status_ = sync())) return status_;
    return status_ = accel_track(line_, r, ACCEL_LAYOUT_AOS, N, (int)st, (int)ed, 1, nullptr, mode, nullptr);
}

void ALine::monitor_print(const double* r, int N, int turn, std::ostream& os) {
    const accel_elem_desc& m = desc_[0];
    if (mon_flag_ == MON_COORD) {
        double ratio = m.f[1];
        int iskip = (int)(1. / ratio);
        if (iskip < 1) iskip = 1;
        if (iskip > N) iskip = N;
        for (int i = 0; i < N; i += iskip) {
            const double* rp = r + 6 * i;
            os << turn << "\t" << rp[0] << "\t" << rp[1] << "\t" << rp[2] << "\t" << rp[3]
               << "\t" << rp[4] << "\t" << rp[5] << std::endl;
        }
    } else if ((mon_flag_ == MON_STAT1 || mon_flag_ == MON_STAT2) && N >= 2) {
        double ar[6], sg[6], cr[6];
        int nl = 0;
        accel_beam_stat(ctx_, r, ACCEL_LAYOUT_AOS, N, ar, sg, cr, &nl);
        os << std::scientific;
        os << turn << "\t" << nl;
        for (int k = 0; k < 6; k++) os << "\t" << ar[k];
        for (int k = 0; k < 6; k++) os << "\t" << sg[k];
        if (mon_flag_ == MON_STAT2)
            for (int k = 0; k < 6; k++) os << "\t" << cr[k];
        os << std::endl;
    }
}

int ALine::pass(double* r, int N) { return pass(r, N, 1); }

int ALine::pass(double* r, int N, int nturn) {
    if ((status_ = sync())) return status_;
    const int ne = (int)desc_.size();
    const bool mon = ne > 0 && desc_[0].type == ACCEL_MONITOR && mon_flag_ != MON_OFF;
    if (!mon)
        return status_ = accel_track(line_, r, ACCEL_LAYOUT_AOS, N, 0, ne, nturn, nullptr, mode, nullptr);
    // AMonitor::pass (accel.cpp:437-475) prints at the start of every interval-th pass
    int interval = std::max(1, (int)desc_[0].f[0]);
    int t = 0;
    while (t < nturn) {
        int c = mon_cnt_pass_ + 1;
        int to_print = ((interval - (c - 1) % interval) % interval);
        if (to_print == 0) {
            mon_cnt_pass_ = c;
            monitor_print(r, N, mon_cnt_pass_ - 1, std::cout);
            int k = std::min(interval, nturn - t);
            status_ = accel_track(line_, r, ACCEL_LAYOUT_AOS, N, 0, ne, k, nullptr, mode, nullptr);
            mon_cnt_pass_ += k - 1;
            t += k;
        } else {
            int k = std::min(to_print, nturn - t);
            status_ = accel_track(line_, r, ACCEL_LAYOUT_AOS, N, 0, ne, k, nullptr, mode, nullptr);
            mon_cnt_pass_ += k;
            t += k;
        }
        if (status_) return status_;
    }
    return status_;
}

int ALine::track_loss(double* r, int N, int nturn, int32_t* loss_turn) {
    if ((status_ = sync())) return status_;
    return status_ = accel_track(line_, r, ACCEL_LAYOUT_AOS, N, 0, (int)desc_.size(), nturn, loss_turn,
                                 mode, nullptr);
}

// ALine::trackDA (aline.cpp:607-715): nray rays x nstep particles, z = 1e-5, the first lost step
// of each ray is its boundary, the area is a triangle fan.
double ALine::trackDA(double xmax, double xmin, double ymax, int nturn, unsigned nray, int nstep,
                      double* rx, double* ry, bool flag_negweight) {
    if (nray < 3) nray = 3;
    if (nray > 51) nray = 51;
    if (nstep < 2) nstep = 2;
    double deltax = xmax - xmin;
    if (deltax < 0) return -1;
    const int np = (int)nray * nstep;
    std::vector<double> xl((size_t)np), yl((size_t)np), r((size_t)6 * np, 0.0);
    for (unsigned i = 0; i < nray; i++)
        for (int j = 0; j < nstep; j++) {
            size_t k = (size_t)i * nstep + j;
            xl[k] = (xmin + deltax * j / (nstep - 1)) * std::cos(i * kPi / (nray - 1));
            yl[k] = (xmin + deltax * j / (nstep - 1)) * std::sin(i * kPi / (nray - 1)) * ymax / xmax;
            r[6 * k + 0] = xl[k];
            r[6 * k + 2] = yl[k];
            r[6 * k + 4] = 1.0e-5;
        }
    std::vector<int32_t> lt((size_t)np, -1);
    if (track_loss(r.data(), np, nturn, lt.data())) return -1;
    for (unsigned i = 0; i < nray; i++) {
        rx[i] = xl[(size_t)i * nstep + nstep - 1];
        ry[i] = yl[(size_t)i * nstep + nstep - 1];
        for (int j = 0; j < nstep; j++)
            if (std::isnan(r[6 * ((size_t)i * nstep + j)])) {
                rx[i] = xl[(size_t)i * nstep + j];
                ry[i] = yl[(size_t)i * nstep + j];
                break;
            }
    }
    double Sxy = 0;
    for (unsigned i = 1; i < nray; i++) {
        double rd1 = std::sqrt(rx[i - 1] * rx[i - 1] + ry[i - 1] * ry[i - 1]);
        double rd2 = std::sqrt(rx[i] * rx[i] + ry[i] * ry[i]);
        double dphi = std::atan2(ry[i], rx[i]) - std::atan2(ry[i - 1], rx[i - 1]);
        if (rx[i] <= 0) Sxy += .5 * rd1 * rd2 * std::sin(dphi);
        else Sxy += (flag_negweight ? .25 : .5) * rd1 * rd2 * std::sin(dphi);
    }
    return Sxy;
}

// ALine::trackMA (aline.cpp:781-836), batched: the ring rotated to each start element is one
// instance of a single batched launch (the reference rotates and tracks one start at a time).
double ALine::trackMA(double dppmax, double dppmin, int nturn, unsigned nstep, double* dpp_plus,
                      double* dpp_minus, unsigned nfam, const unsigned* lfam) {
    if (nfam == 0) return 0;
    const int per = 2 * ((int)nstep + 1);
    const double stepsize = (dppmax - dppmin) / nstep;
    std::vector<accel_line*> lines(nfam, nullptr);
    std::vector<double> soa((size_t)6 * per * nfam, 0.0);
    const int64_t ntot = (int64_t)per * nfam;
    std::vector<int64_t> off(nfam + 1);
    for (unsigned i = 0; i <= nfam; i++) off[i] = (int64_t)i * per;
    for (unsigned i = 0; i < nfam; i++) {
        std::vector<accel_elem_desc> rot = desc_;
        std::rotate(rot.begin(), rot.begin() + (lfam[i] % rot.size()), rot.end());
        if ((status_ = accel_line_create(ctx_, rot.data(), (int)rot.size(), &lines[i]))) break;
        for (int j = 0; j < (int)nstep + 1; j++) {
            soa[(size_t)5 * ntot + (size_t)i * per + 2 * j] = dppmin + stepsize * j;
            soa[(size_t)5 * ntot + (size_t)i * per + 2 * j + 1] = -(dppmin + stepsize * j);
        }
    }
    double avg = 0;
    accel::DevBuf d_soa;  // counted against the library's device-memory limit
    int ast = status_ ? status_ : d_soa.ensure(soa.size() * sizeof(double));
    if (!status_ && !ast) {
        cudaMemcpy(d_soa.p, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice);
        status_ = accel_track_batched(lines.data(), (int)nfam, off.data(), (double*)d_soa.p, ntot, nturn, nullptr, mode,
                                      nullptr);
        cudaDeviceSynchronize();
        cudaMemcpy(soa.data(), d_soa.p, sizeof(double) * (size_t)ntot, cudaMemcpyDeviceToHost);  // x row
        d_soa.release();
        for (unsigned i = 0; i < nfam; i++) {
            dpp_plus[i] = dppmin;
            dpp_minus[i] = -dppmin;
            for (int j = 1; j < (int)nstep + 1; j++) {
                if (!std::isnan(soa[(size_t)i * per + 2 * j])) dpp_plus[i] = dppmin + stepsize * j;
                if (!std::isnan(soa[(size_t)i * per + 2 * j + 1])) dpp_minus[i] = -(dppmin + stepsize * j);
            }
            avg += std::fmin(dpp_plus[i], -dpp_minus[i]);
        }
        avg /= nfam;
    } else if (!status_) {
        status_ = ast;
    }
    for (accel_line* l : lines)
        if (l) accel_line_destroy(l);
    return avg;
}

// ---- turn-by-turn tunes -------------------------------------------------------------------------
// r: AoS particles; x and y of every particle before each of nt turns into xs[p * nt + t],
// ys[p * nt + t] (a lost particle records NaN from then on)
static int record_tbt(ALine& L, std::vector<double>& r, int np, unsigned nt, std::vector<double>& xs,
                      std::vector<double>& ys) {
    xs.assign((size_t)np * nt, 0.0);
    ys.assign((size_t)np * nt, 0.0);
    for (unsigned t = 0; t < nt; t++) {
        for (int p = 0; p < np; p++) {
            xs[(size_t)p * nt + t] = r[(size_t)6 * p];
            ys[(size_t)p * nt + t] = r[(size_t)6 * p + 2];
        }
        if (t + 1 < nt) {
            int s = L.pass(r.data(), np, 0, L.getnumber());
            if (s) return s;
        }
    }
    return ACCEL_OK;
}

void ALine::tracktune(double& tunex, double& tuney, unsigned nturn, double x0, double y0, double xlow,
                      double xhi, double ylow, double yhi) {
    const unsigned nt = pow2_at_least(nturn);
    std::vector<double> r(6, 0.0), xs, ys;
    r[0] = x0;
    r[2] = y0;
    if ((status_ = record_tbt(*this, r, 1, nt, xs, ys))) { tunex = tuney = NAN; return; }
    tunex = naff((int)nt, xs.data(), xlow, xhi);
    tuney = naff((int)nt, ys.data(), ylow, yhi);
}

double ALine::trackDiffusion(int nturn, unsigned np, const double* x0, const double* y0, double* nux,
                             double* nuy, double* dif, double xlow, double xhi, double ylow, double yhi) {
    const unsigned nt = pow2_at_least((unsigned)std::max(1, nturn));
    const double mdiffu = -4 * std::log(nt * 1.0);
    std::vector<double> r((size_t)6 * np, 0.0), xs, ys;
    for (unsigned p = 0; p < np; p++) { r[(size_t)6 * p] = x0[p]; r[(size_t)6 * p + 2] = y0[p]; }
    if ((status_ = record_tbt(*this, r, (int)np, nt, xs, ys))) return NAN;
    double tdif = 0;
    const int h = (int)(nt >> 1);
    for (unsigned p = 0; p < np; p++) {
        const double* xl = xs.data() + (size_t)p * nt;
        const double* yl = ys.data() + (size_t)p * nt;
        if (std::isnan(xl[nt - 1])) {
            nux[p] = nuy[p] = dif[p] = NAN;
            tdif += -3.0;
            continue;
        }
        const double nux0 = naff(h, xl, xlow, xhi), nuy0 = naff(h, yl, ylow, yhi);
        const double nux1 = naff(h, xl + h, xlow, xhi), nuy1 = naff(h, yl + h, ylow, yhi);
        nux[p] = nux0;
        nuy[p] = nuy0;
        const double d = std::hypot(nux1 - nux0, nuy1 - nuy0);
        dif[p] = std::max(mdiffu, std::log(d * 2.0 / nt));
        tdif += dif[p];
    }
    return tdif;
}

void ALine::trackdnudexy(double* dnudexy, unsigned nturn, double xm, double ym, std::ostream* log) {
    Twiss tw;
    calctwiss(tw);
    const double tunex = tw.psix / 2 / kPi, tuney = tw.psiy / 2 / kPi;
    const int np = 6;
    const double tiny = 1.0e-5;
    const unsigned nt = pow2_at_least(nturn);
    // 6 horizontal amplitudes, then 6 vertical ones, tracked together
    std::vector<double> r((size_t)6 * 2 * np, 0.0), de(2 * np), xs, ys;
    for (int k = 0; k < np; k++) {
        double* a = &r[(size_t)6 * k];
        a[0] = tiny + k * 1.0 / (np - 1) * xm;
        a[2] = tiny + a[0] * .02;
        de[k] = a[0] * a[0] / tw.betx;
        double* b = &r[(size_t)6 * (np + k)];
        b[2] = tiny + k * 1.0 / (np - 1) * ym;
        b[0] = tiny + b[2] * .02;
        de[np + k] = b[2] * b[2] / tw.bety;
    }
    for (int q = 0; q < 4; q++) dnudexy[q] = NAN;
    if ((status_ = record_tbt(*this, r, 2 * np, nt, xs, ys))) return;
    std::vector<double> xt(2 * np), yt(2 * np);
    for (int k = 0; k < 2 * np; k++) {
        xt[k] = naff((int)nt, xs.data() + (size_t)k * nt, std::max(0.0, tunex - 0.1), std::min(0.5, tunex + 0.1));
        yt[k] = naff((int)nt, ys.data() + (size_t)k * nt, std::max(0.0, tuney - 0.1), std::min(0.5, tuney + 0.1));
        if (log) *log << de[k] << "\t" << xt[k] << "\t" << yt[k] << std::endl;
    }
    fit_slope(np, de.data(), xt.data(), dnudexy[0]);
    fit_slope(np, de.data(), yt.data(), dnudexy[1]);
    fit_slope(np, de.data() + np, xt.data() + np, dnudexy[2]);
    fit_slope(np, de.data() + np, yt.data() + np, dnudexy[3]);
}

// ---- optics --------------------------------------------------------------------------------------
int ALine::getm66(double* m, unsigned st, unsigned ed, double dpp, double delta, bool exact) {
    if ((status_ = sync())) return status_;
    return status_ = accel_m66(line_, (int)st, (int)ed, dpp, delta, exact ? 0 : 1, m);
}

int ALine::getco4(double* rc, double dp, double delta) {
    set_rad_onoff(0);
    set_cavity_onoff(false);
    double m[36];
    if (getm66(m, dp, delta)) return status_;
    double r[6] = {0, 0, 0, 0, 0, dp};
    if (pass(r, 1, 0, getnumber())) return status_;
    if (!solve_I_minus(m, 4, r, rc)) return status_ = ACCEL_E_INVALID;
    return ACCEL_OK;
}

int ALine::getco6(double* rc, double delta) {
    set_rad_onoff(1);
    set_cavity_onoff(true);
    double m[36];
    if (getm66(m, 0., delta)) return status_;
    double r[6] = {0, 0, 0, 0, 0, 0};
    if (pass(r, 1, 0, getnumber())) return status_;
    if (!solve_I_minus(m, 6, r, rc)) return status_ = ACCEL_E_INVALID;
    return ACCEL_OK;
}

void ALine::calctune(double& tunex, double& tuney, double dp, double delta) {
    double m[36];
    getm66(m, dp, delta);
    tunex = tune_of(m, 0);
    tuney = tune_of(m, 2);
}

void ALine::calctwiss(Twiss& tw, double dp, double delta) {
    double m[36];
    getm66(m, dp, delta);
    tw.s = 0;
    tw.psix = std::acos((m[0] + m[7]) * 0.5);
    tw.psiy = std::acos((m[14] + m[21]) * 0.5);
    tw.betx = m[1] / std::sin(tw.psix);
    tw.bety = m[15] / std::sin(tw.psiy);
    tw.alfx = (m[0] - m[7]) / std::sin(tw.psix) / 2.0;
    tw.alfy = (m[14] - m[21]) / std::sin(tw.psiy) / 2.0;
}

// Twiss at a list of elements (aline.cpp:1044-1091)
void ALine::calctwiss(Twiss* tw, const unsigned* indx, int n, double dp, double delta) {
    Twiss tw0;
    calctwiss(tw0, dp, delta);
    tw0.psix = tw0.psiy = 0;
    double T[36];
    unsigned id = indx[0];
    getm66(T, 0, id, dp, delta);
    double len01 = getlength(0, id);
    for (int i = 0; i < n; i++) {
        Twiss t1;
        t1.s = tw0.s + len01;
        auto M = [&](int a, int b) { return T[6 * (a - 1) + (b - 1)]; };
        t1.betx = 1.0 / tw0.betx * (std::pow(M(1, 1) * tw0.betx - M(1, 2) * tw0.alfx, 2) + std::pow(M(1, 2), 2));
        t1.bety = 1.0 / tw0.bety * (std::pow(M(3, 3) * tw0.bety - M(3, 4) * tw0.alfy, 2) + std::pow(M(3, 4), 2));
        t1.alfx = -1.0 / tw0.betx * ((M(1, 1) * tw0.betx - M(1, 2) * tw0.alfx) * (M(2, 1) * tw0.betx - M(2, 2) * tw0.alfx) + M(1, 2) * M(2, 2));
        t1.alfy = -1.0 / tw0.bety * ((M(3, 3) * tw0.bety - M(3, 4) * tw0.alfy) * (M(4, 3) * tw0.bety - M(4, 4) * tw0.alfy) + M(3, 4) * M(4, 4));
        t1.psix = tw0.psix + std::atan2(M(1, 2), M(1, 1) * tw0.betx - M(1, 2) * tw0.alfx);
        t1.psiy = tw0.psiy + std::atan2(M(3, 4), M(3, 3) * tw0.bety - M(3, 4) * tw0.alfy);
        tw[i] = t1;
        tw0 = t1;
        if (i < n - 1) {
            unsigned id2 = indx[i + 1];
            getm66(T, id, id2, dp, delta);
            len01 = getlength(id, id2);
            id = id2;
        }
    }
}

void ALine::calcchrom2(double& chromx, double& chromy, double& chromx2, double& chromy2) {
    const int np = 11;
    double sx = 0, sxx = 0, sy[2] = {0, 0}, sxy[2] = {0, 0};
    for (int i = 0; i < np; i++) {
        double dpp = 1.0e-3 * (i - 6.0), c[2];
        calcchrom(c[0], c[1], dpp);
        sx += dpp;
        sxx += dpp * dpp;
        for (int p = 0; p < 2; p++) {
            sy[p] += c[p];
            sxy[p] += dpp * c[p];
        }
    }
    const double den = np * sxx - sx * sx;
    chromx2 = (np * sxy[0] - sx * sy[0]) / den / 2.0;
    chromy2 = (np * sxy[1] - sx * sy[1]) / den / 2.0;
    calcchrom(chromx, chromy, 0);
}

void ALine::calcchrom(double& chromx, double& chromy, double dp, double delta) {
    const double dpp = 1.0e-5;
    double tx0, ty0, tx, ty;
    calctune(tx0, ty0, dp - dpp, delta);
    calctune(tx, ty, dp + dpp, delta);
    chromx = (tx - tx0) / dpp / 2.0;
    chromy = (ty - ty0) / dpp / 2.0;
}

void ALine::knob_add(unsigned nfam, const unsigned* lfam, int order, double dv) {
    for (unsigned j = 0; j < nfam; j++) {
        accel_elem_desc& d = desc_[lfam[j]];
        if (d.type == ACCEL_QUAD && order == 1) d.f[0] += dv;
        else if (d.type == ACCEL_STRMPOLE) d.poly_b[order] += dv;
    }
    dirty_ = true;
}

// ALine::correcttune / correctchrom (aline.cpp:1187-1418): a 2x2 response from +1e-5 steps of
// each family, then one linear step toward the target.
void ALine::correcttune(double& tunex, double& tuney, unsigned nfam1, unsigned nfam2,
                        const unsigned* lfam1, const unsigned* lfam2) {
    double tx0, ty0, resp[2][2];
    calctune(tx0, ty0);
    const double delta = 1.0e-5;
    const unsigned* lf[2] = {lfam1, lfam2};
    unsigned nf[2] = {nfam1, nfam2};
    for (int i = 0; i < 2; i++) {
        knob_add(nf[i], lf[i], 1, delta);
        double tx, ty;
        calctune(tx, ty);
        resp[i][0] = (tx - tx0) / delta;
        resp[i][1] = (ty - ty0) / delta;
        knob_add(nf[i], lf[i], 1, -delta);
    }
    double detr = resp[0][0] * resp[1][1] - resp[0][1] * resp[1][0];
    double d1 = -(resp[1][1] * (tx0 - tunex) - resp[1][0] * (ty0 - tuney)) / detr;
    double d2 = -(-resp[0][1] * (tx0 - tunex) + resp[0][0] * (ty0 - tuney)) / detr;
    knob_add(nfam1, lfam1, 1, d1);
    knob_add(nfam2, lfam2, 1, d2);
    calctune(tunex, tuney);
}

void ALine::correctchrom(double& chromx, double& chromy, unsigned nfam1, unsigned nfam2,
                         const unsigned* lfam1, const unsigned* lfam2) {
    double cx0, cy0, resp[2][2];
    calcchrom(cx0, cy0);
    const double delta = 1.0e-5;
    const unsigned* lf[2] = {lfam1, lfam2};
    unsigned nf[2] = {nfam1, nfam2};
    for (int i = 0; i < 2; i++) {
        knob_add(nf[i], lf[i], 2, delta);
        double cx, cy;
        calcchrom(cx, cy);
        resp[i][0] = (cx - cx0) / delta;
        resp[i][1] = (cy - cy0) / delta;
        knob_add(nf[i], lf[i], 2, -delta);
    }
    double detr = resp[0][0] * resp[1][1] - resp[0][1] * resp[1][0];
    double d1 = -(resp[1][1] * (cx0 - chromx) - resp[1][0] * (cy0 - chromy)) / detr;
    double d2 = -(-resp[0][1] * (cx0 - chromx) + resp[0][0] * (cy0 - chromy)) / detr;
    knob_add(nfam1, lfam1, 2, d1);
    knob_add(nfam2, lfam2, 2, d2);
    calcchrom(chromx, chromy);
}

// Newton on exact one-turn matrices: the tunes from the tangent map about (0, 0, 0, 0, 0, dp),
// the point the reference's calctune expands about (no delta-difference noise), and their 2 x 2
// response to the two families from the exact knob derivative of that matrix (accel_m66_knob:
// hyper-dual numbers through every element, no difference in the knobs), iterated until the
// residual stops shrinking.  Returns the iterations used.
static void exact_tunes(ALine& L, double& tx, double& ty, double dp) {
    double m[36];
    L.getm66(m, 0, L.getnumber(), dp, 1e-8, true);
    tx = tune_of(m, 0);
    ty = tune_of(m, 2);
}

// The coefficients knob_add moves for a family at multipole `order`: Quad K (order 1) or
// StrMPole PolynomB[order].
static void family_coeffs(const ALine& L, unsigned nfam, const unsigned* lfam, int order, std::vector<int32_t>& e,
                          std::vector<int32_t>& f, std::vector<int32_t>& i) {
    e.clear(); f.clear(); i.clear();
    for (unsigned j = 0; j < nfam; j++) {
        const accel_elem_desc& d = L.element(lfam[j]);
        if (d.type == ACCEL_QUAD && order == 1) { e.push_back((int32_t)lfam[j]); f.push_back(ACCEL_F_K); i.push_back(0); }
        else if (d.type == ACCEL_STRMPOLE) { e.push_back((int32_t)lfam[j]); f.push_back(ACCEL_F_POLYNOMB); i.push_back(order); }
    }
}

// Exact tunes at dp and J[k][i] = d tune_k / d family_i: tune = acos(c) / 2 pi with
// c = (m_kk + m_k+1,k+1) / 2, so d tune = -dc / (2 pi sqrt(1 - c^2)).
static int tune_response(ALine& L, double dp, int order, const unsigned* nf, const unsigned* const* lf,
                         double t[2], double J[2][2]) {
    const double r0[6] = {0, 0, 0, 0, 0, dp};
    accel_line* line = L.device_line();
    if (!line) return L.last_status() ? L.last_status() : ACCEL_E_INVALID;
    for (int i = 0; i < 2; i++) {
        std::vector<int32_t> e, f, x;
        family_coeffs(L, nf[i], lf[i], order, e, f, x);
        if (e.empty()) return accel::fail(ACCEL_E_INVALID, "a correction family has no magnet the knob can move");
        double m[36], dm[36];
        int s = accel_m66_knob(line, 0, (int)L.getnumber(), r0, (int)e.size(), e.data(), f.data(), x.data(), m, dm);
        if (s) return s;
        for (int k = 0; k < 2; k++) {
            const int p = 2 * k;
            const double c = 0.5 * (m[6 * p + p] + m[6 * (p + 1) + p + 1]);
            const double dc = 0.5 * (dm[6 * p + p] + dm[6 * (p + 1) + p + 1]);
            t[k] = tune_of(m, p);
            J[k][i] = -dc / (2.0 * kPi * std::sqrt(1.0 - c * c));
        }
    }
    return ACCEL_OK;
}

int ALine::correct_tune_exact(double& tunex, double& tuney, unsigned nfam1, unsigned nfam2,
                              const unsigned* lfam1, const unsigned* lfam2, int maxit) {
    const double tgt[2] = {tunex, tuney};
    const unsigned* lf[2] = {lfam1, lfam2};
    unsigned nf[2] = {nfam1, nfam2};
    int it = 0;
    for (; it < maxit; it++) {
        double t0[2], J[2][2];
        if ((status_ = tune_response(*this, 0.0, 1, nf, lf, t0, J))) return it;
        double res = std::hypot(t0[0] - tgt[0], t0[1] - tgt[1]);
        if (res < 1e-12) break;
        double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        double r0 = tgt[0] - t0[0], r1 = tgt[1] - t0[1];
        knob_add(nfam1, lfam1, 1, (J[1][1] * r0 - J[0][1] * r1) / det);
        knob_add(nfam2, lfam2, 1, (-J[1][0] * r0 + J[0][0] * r1) / det);
    }
    exact_tunes(*this, tunex, tuney, 0);
    return it;
}

// Chromaticity as the reference's calcchrom defines it, the tune change over dpp = +-1e-5
// (aline.cpp:1108-1158), here from exact tunes; its knob response from the exact knob
// derivatives of those tunes.
static const double kChromDpp = 1.0e-5;

static void exact_chrom(ALine& L, double& cx, double& cy) {
    double a0, a1, b0, b1;
    exact_tunes(L, a0, a1, -kChromDpp);
    exact_tunes(L, b0, b1, kChromDpp);
    cx = (b0 - a0) / kChromDpp / 2.0;
    cy = (b1 - a1) / kChromDpp / 2.0;
}

int ALine::correct_chrom_exact(double& chromx, double& chromy, unsigned nfam1, unsigned nfam2,
                               const unsigned* lfam1, const unsigned* lfam2, int maxit) {
    const double tgt[2] = {chromx, chromy};
    const unsigned* lf[2] = {lfam1, lfam2};
    unsigned nf[2] = {nfam1, nfam2};
    int it = 0;
    double prev = 1e300;
    for (; it < maxit; it++) {
        double tm[2], tp[2], Jm[2][2], Jp[2][2];
        if ((status_ = tune_response(*this, -kChromDpp, 2, nf, lf, tm, Jm))) return it;
        if ((status_ = tune_response(*this, kChromDpp, 2, nf, lf, tp, Jp))) return it;
        double c0[2], J[2][2];
        for (int k = 0; k < 2; k++) {
            c0[k] = (tp[k] - tm[k]) / kChromDpp / 2.0;
            for (int i = 0; i < 2; i++) J[k][i] = (Jp[k][i] - Jm[k][i]) / kChromDpp / 2.0;
        }
        double res = std::hypot(c0[0] - tgt[0], c0[1] - tgt[1]);
        if (res < 1e-9 || res >= prev) break;
        prev = res;
        double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        double r0 = tgt[0] - c0[0], r1 = tgt[1] - c0[1];
        knob_add(nfam1, lfam1, 2, (J[1][1] * r0 - J[0][1] * r1) / det);
        knob_add(nfam2, lfam2, 2, (-J[1][0] * r0 + J[0][0] * r1) / det);
    }
    exact_chrom(*this, chromx, chromy);
    return it;
}

}  // namespace accelgpu

extern "C" int accel_naff(const double* data, int n, double xlow, double xhi, double* nu) {
    if (!data || !nu || n < 4) return accel::fail(ACCEL_E_INVALID, "accel_naff: need data, nu and n >= 4");
    *nu = accelgpu::naff(n, data, xlow, xhi);
    return ACCEL_OK;
}

// ALine::trackDiffusion and ALine::tracktune (aline.cpp:716-779, 1159-1186) on a line of the C
// ABI: the points are tracked together on the device one turn per call (the line's descriptors in
// a host ALine on the same context), the NAFF analysis runs on the host.
extern "C" int accel_track_diffusion(accel_line* L, int nturn, int np, const double* x0, const double* y0,
                                     double* nux, double* nuy, double* dif, double xlow, double xhi,
                                     double ylow, double yhi, int mode, double* total) {
    if (!L || np <= 0 || nturn < 2 || !x0 || !y0 || !nux || !nuy || !dif)
        return accel::fail(ACCEL_E_INVALID, "accel_track_diffusion: need a line, np > 0, nturn >= 2 and every array");
    if (mode != ACCEL_MODE_FUSED && mode != ACCEL_MODE_PLAIN && mode != ACCEL_MODE_EXACT)
        return accel::fail(ACCEL_E_INVALID, "accel_track_diffusion: bad mode");
    accelgpu::ALine a(L->ctx, L->desc);
    a.mode = mode;
    const double t = a.trackDiffusion(nturn, (unsigned)np, x0, y0, nux, nuy, dif, xlow, xhi, ylow, yhi);
    if (a.last_status()) return a.last_status();
    if (total) *total = t;
    return ACCEL_OK;
}

extern "C" int accel_track_tune(accel_line* L, int nturn, double x0, double y0, double xlow, double xhi,
                                double ylow, double yhi, int mode, double* tunex, double* tuney) {
    if (!L || nturn < 4 || !tunex || !tuney)
        return accel::fail(ACCEL_E_INVALID, "accel_track_tune: need a line, nturn >= 4, tunex and tuney");
    if (mode != ACCEL_MODE_FUSED && mode != ACCEL_MODE_PLAIN && mode != ACCEL_MODE_EXACT)
        return accel::fail(ACCEL_E_INVALID, "accel_track_tune: bad mode");
    accelgpu::ALine a(L->ctx, L->desc);
    a.mode = mode;
    a.tracktune(*tunex, *tuney, (unsigned)nturn, x0, y0, xlow, xhi, ylow, yhi);
    return a.last_status();
}

// ALine::correcttune / correctchrom (aline.cpp:1243-1418) on a line of the C ABI.  method 0: Newton
// iterations driven by exact knob derivatives (accel_m66_knob) until the residual is below 1e-12
// (tunes) or 1e-9 (chromaticities) or stops shrinking, at most maxit; method 1: the reference's
// fit, one step of a response built by stepping each family by 1e-5.  The families' coefficients
// are written back to the line.
static int correct_on_line(accel_line* L, const int32_t* fam1, int n1, const int32_t* fam2, int n2,
                           double* a, double* b, int method, int maxit, int* iterations, bool chrom) {
    if (!L || !fam1 || !fam2 || n1 <= 0 || n2 <= 0 || !a || !b || (method != 0 && method != 1) || maxit < 1)
        return accel::fail(ACCEL_E_INVALID, "bad argument");
    const int ne = (int)L->desc.size();
    std::vector<unsigned> l1((size_t)n1), l2((size_t)n2);
    for (int j = 0; j < n1; j++) {
        if (fam1[j] < 0 || fam1[j] >= ne) return accel::fail(ACCEL_E_INVALID, "family element out of range");
        l1[(size_t)j] = (unsigned)fam1[j];
    }
    for (int j = 0; j < n2; j++) {
        if (fam2[j] < 0 || fam2[j] >= ne) return accel::fail(ACCEL_E_INVALID, "family element out of range");
        l2[(size_t)j] = (unsigned)fam2[j];
    }
    accelgpu::ALine line(L->ctx, L->desc);
    int it = 1;
    if (method == 0) {
        it = chrom ? line.correct_chrom_exact(*a, *b, (unsigned)n1, (unsigned)n2, l1.data(), l2.data(), maxit)
                   : line.correct_tune_exact(*a, *b, (unsigned)n1, (unsigned)n2, l1.data(), l2.data(), maxit);
    } else if (chrom) {
        line.correctchrom(*a, *b, (unsigned)n1, (unsigned)n2, l1.data(), l2.data());
    } else {
        line.correcttune(*a, *b, (unsigned)n1, (unsigned)n2, l1.data(), l2.data());
    }
    if (line.last_status()) return line.last_status();
    L->desc = line.descs();
    L->dirty = true;
    if (iterations) *iterations = it;
    return ACCEL_OK;
}

extern "C" int accel_correct_tune(accel_line* L, const int32_t* fam1, int n1, const int32_t* fam2, int n2,
                                  double* tunex, double* tuney, int method, int maxit, int* iterations) {
    return correct_on_line(L, fam1, n1, fam2, n2, tunex, tuney, method, maxit, iterations, false);
}

extern "C" int accel_correct_chrom(accel_line* L, const int32_t* fam1, int n1, const int32_t* fam2, int n2,
                                   double* chromx, double* chromy, int method, int maxit, int* iterations) {
    return correct_on_line(L, fam1, n1, fam2, n2, chromx, chromy, method, maxit, iterations, true);
}
