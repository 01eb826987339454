// host_aline.hpp — the reference's ALine interface (accel.h:587-657) over the GPU C-ABI.
//
// A drop-in for code written against the reference's ALine: the same pass / trackDA / trackMA /
// getm66 / getco / calctune / calcchrom / correcttune / correctchrom / setrfphase / set_*_onoff /
// findelements / resetfirstelement / serialize entry points, with the lattice held as host
// descriptors and every particle pass running on the device.  Monitor printing (AMonitor::pass,
// accel.cpp:437-475) happens on the host between device segments.
#pragma once
#include <cstdint>
#include <iosfwd>
#include <string>
#include <vector>
#include "accel_gpu.h"

namespace accelgpu {

struct Twiss {  // reference struct Twiss, accel.h:669-676
    double s = 0, psix = 0, psiy = 0, betx = 0, alfx = 0, bety = 0, alfy = 0;
    void serialize(std::ostream& os) const;
};

// Monitor print flags (AMonitor::flag_print, accel.h:132)
enum MonitorFlag : unsigned { MON_OFF = 0, MON_COORD = 1, MON_STAT1 = 2, MON_STAT2 = 3 };

class ALine {
public:
    static ALine* load(const std::string& path, accel_ctx* ctx, int* status = nullptr);
    static ALine* deserialize(std::istream& is, accel_ctx* ctx, int* status = nullptr);
    ALine(accel_ctx* ctx, std::vector<accel_elem_desc> elems);
    ~ALine();
    ALine(const ALine&) = delete;
    ALine& operator=(const ALine&) = delete;

    // structure (aline.cpp:126-219, 520-605)
    unsigned getnumber() const { return (unsigned)desc_.size(); }
    double getlength() const { return getlength(0, getnumber()); }
    double getlength(unsigned ed) const { return getlength(0, ed); }
    double getlength(unsigned st, unsigned ed) const;
    accel_elem_desc& element(unsigned i) { dirty_ = true; return desc_.at(i); }
    const accel_elem_desc& element(unsigned i) const { return desc_.at(i); }
    int addelement(const accel_elem_desc& e);
    int insertelement(unsigned i, const accel_elem_desc& e);
    int deleteelement(unsigned i);
    unsigned findelements(unsigned* list, const std::string& type, const std::string& famname,
                          unsigned index = 0) const;
    unsigned findelements(unsigned* list, const std::string& type) const;
    unsigned resetfirstelement(unsigned eindex);
    unsigned resetfirstelement(const std::string& type, const std::string& famname, unsigned index = 1);
    void serialize(std::ostream& os, int precision = 6) const;

    // switches (aline.cpp:220-293, 410-518)
    int setenergy(double en);
    double setrfphase();
    double setrfphase(double phis);
    int set_rad_onoff(unsigned flag);
    int set_cavity_onoff(bool flag);
    int set_wake_onoff(bool flag);
    int set_crab_onoff(bool flag);
    int set_monitor(unsigned flag, unsigned index = 0);
    int set_monitor_pass(int num = 0);
    unsigned monitor_flag() const { return mon_flag_; }
    // one AMonitor print (coordinates of every 1/ratio-th particle, or beam statistics) labelled turn
    void monitor_print(const double* r, int N, int turn, std::ostream& os);

    // fields by the reference's names (AccelElement::setfield/getfield)
    int setfield(unsigned idx, const std::string& name, double value, unsigned index = 0);
    int getfield(unsigned idx, const std::string& name, double* value, unsigned index = 0) const;

    // tracking (aline.cpp:313-363, 607-836)
    int pass(double* r, int N, unsigned st, unsigned ed);
    int pass(double* r, int N);
    int pass(double* r, int N, int nturn);
    int track_loss(double* r, int N, int nturn, int32_t* loss_turn);
    double trackDA(double xmax, double xmin, double ymax, int nturn, unsigned nray, int nstep,
                   double* rx, double* ry, bool flag_negweight = false);
    double trackMA(double dppmax, double dppmin, int nturn, unsigned nstep, double* dpp_plus,
                   double* dpp_minus, unsigned nfam, const unsigned* lfam);

    // optics (aline.cpp:838-1418); exact = tangent map instead of the delta difference
    int getm66(double* m, unsigned st, unsigned ed, double dpp = 0, double delta = 1e-8,
               bool exact = false);
    int getm66(double* m, double dpp = 0, double delta = 1e-8, bool exact = false) {
        return getm66(m, 0, getnumber(), dpp, delta, exact);
    }
    int getco4(double* rc4, double dp = 0, double delta = 1e-8);
    int getco6(double* rc6, double delta = 1e-8);
    void calctune(double& tunex, double& tuney, double dp = 0, double delta = 1e-8);
    void calctwiss(Twiss& tw, double dp = 0, double delta = 1e-8);
    void calctwiss(Twiss* tw, const unsigned* indx, int n, double dp = 0, double delta = 1e-8);
    void calcchrom(double& chromx, double& chromy, double dp = 0, double delta = 1e-8);
    // second-order chromaticity: half the least-squares slope of the chromaticity over the 11
    // momentum offsets 1e-3 * (i - 6), i = 0..10 (aline.cpp:1127-1158)
    void calcchrom2(double& chromx, double& chromy, double& chromx2, double& chromy2);

    // turn-by-turn tunes (aline.cpp:1159-1185, 716-779, 1421-1500).  Particles are tracked
    // together on the device, one turn per call, their x and y recorded before every turn; the
    // record length is nturn rounded up to a power of two, as the reference does.
    void tracktune(double& tunex, double& tuney, unsigned nturn, double x0, double y0,
                   double xlow = 0, double xhi = 0.5, double ylow = 0, double yhi = 0.5);
    double trackDiffusion(int nturn, unsigned np, const double* x0, const double* y0, double* nux,
                          double* nuy, double* dif, double xlow = 0, double xhi = 0.5,
                          double ylow = 0, double yhi = 0.5);
    // amplitude-dependent tune shift: dnux/dex, dnuy/dex, dnux/dey, dnuy/dey (slopes of the tunes
    // at 6 amplitudes against 2J = x^2/beta); per-amplitude lines "2J  nux  nuy" go to `log`
    void trackdnudexy(double* dnudexy, unsigned nturn, double xm, double ym, std::ostream* log = nullptr);
    // one difference-response step, as the reference (aline.cpp:1243-1418)
    void correcttune(double& tunex, double& tuney, unsigned nfam1, unsigned nfam2,
                     const unsigned* lfam1, const unsigned* lfam2);
    void correctchrom(double& chromx, double& chromy, unsigned nfam1, unsigned nfam2,
                      const unsigned* lfam1, const unsigned* lfam2);
    // Newton iterations on exact one-turn matrices (tangent maps), to convergence
    int correct_tune_exact(double& tunex, double& tuney, unsigned nfam1, unsigned nfam2,
                           const unsigned* lfam1, const unsigned* lfam2, int maxit = 8);
    int correct_chrom_exact(double& chromx, double& chromy, unsigned nfam1, unsigned nfam2,
                            const unsigned* lfam1, const unsigned* lfam2, int maxit = 8);

    accel_line* device_line();  // synced accel_line (rebuilt after host edits)
    const std::vector<accel_elem_desc>& descs() const { return desc_; }
    accel_ctx* ctx() const { return ctx_; }
    int last_status() const { return status_; }
    int mode = ACCEL_MODE_FUSED;

private:
    int sync();
    void knob_add(unsigned nfam, const unsigned* lfam, int order, double dv);
    accel_ctx* ctx_;
    std::vector<accel_elem_desc> desc_;
    accel_line* line_ = nullptr;
    bool dirty_ = true;
    int status_ = ACCEL_OK;
    int mon_cnt_pass_ = 0;
    unsigned mon_flag_ = MON_OFF;
};

double tune_of(const double* m, int plane);  // acos((m_kk + m_k+1,k+1)/2) / 2 pi
// Fundamental frequency of a real turn-by-turn record (the reference's naff, utility.cpp:21-97):
// the largest spectral line with frequency in [xlow, xhi] (bins of 1/N), then the maximum of the
// sin^4-windowed projection |sum_i X_i w_i exp(-2 pi i nu i)| within one bin of it, by golden-
// section search to 3e-8 relative.
double naff(int N, const double* X, double xlow = 0, double xhi = 0.5);
const char* elem_type_name(int type);        // the reference's class name: "Drift", "StrMPole", ...

}  // namespace accelgpu
