/* accel_oracle.c — TEST INFRASTRUCTURE ONLY: CPU oracle for the Accel+ tracking path.
 *
 * A restatement, in plain C over accel_elem_desc descriptors, of the reference's integrators
 * (src/lib/accel/atpass.cpp) and element passes (src/lib/accel/accel.cpp).  Each function cites
 * the reference lines it follows.  Arithmetic keeps the reference's operation order (built with
 * -ffp-contract=off it is bit-identical to the reference library; the tests check that against
 * oracle/_ref and tests/golden).  The product never loads this file's library: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg do, as the checker.
 *
 * Parts with no reference counterpart, restated from the physics and marked "NEW":
 *   the longitudinal broadband-resonator wake (ACCEL_LONGWAKE) and the Gaussian source used for
 *   quantum excitation (the reference uses a racy rand()-based Box-Muller, utility.cpp:194-217).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "accel_oracle.h"

#define O_PI     3.1415926535897932384626
#define O_TWOPI  (2 * O_PI)
#define O_C0     2.99792458e8
#define O_CGAMMA 8.846056192e-05
/* Yoshida 4th-order split constants, accel.h:44-47 */
#define O_DRIFT1  0.6756035959798286638
#define O_DRIFT2 -0.1756035959798286639
#define O_KICK1   1.351207191959657328
#define O_KICK2  -1.702414383919314656
#define O_SQR(X) ((X) * (X))

/* ------------------------------------------------------------------------------------------ */
/* Gaussian source (NEW; statistical parity only)                                               */
/* ------------------------------------------------------------------------------------------ */
static uint64_t splitmix(uint64_t* x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
void orc_rng_seed(orc_rng* g, uint64_t seed) {
    uint64_t x = seed;
    g->s[0] = splitmix(&x);
    g->s[1] = splitmix(&x);
    g->have = 0;
    g->spare = 0.0;
}
static double orc_uniform(orc_rng* g) { /* xorshift128+, 53-bit mantissa in (0,1) */
    uint64_t s1 = g->s[0];
    const uint64_t s0 = g->s[1];
    g->s[0] = s0;
    s1 ^= s1 << 23;
    g->s[1] = s1 ^ s0 ^ (s1 >> 18) ^ (s0 >> 5);
    uint64_t v = g->s[1] + s0;
    return ((double)(v >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
double orc_gauss(orc_rng* g) { /* Box-Muller, both outputs used */
    if (g->have) { g->have = 0; return g->spare; }
    double u1 = orc_uniform(g), u2 = orc_uniform(g);
    double rad = sqrt(-2.0 * log(u1));
    g->spare = rad * sin(O_TWOPI * u2);
    g->have = 1;
    return rad * cos(O_TWOPI * u2);
}

/* ------------------------------------------------------------------------------------------ */
/* Integrators on one particle (atpass.cpp)                                                    */
/* ------------------------------------------------------------------------------------------ */

/* atpass.cpp:6-13 — kept with its path-length term SQR(px + SQR(y)), which uses the already
 * advanced y; reached only from the K == 0 branch of the linear quad. */
static void o_drift(double* r, double L) {
    double p_norm = 1.0 / (1 + r[5]);
    r[0] += r[1] * L;
    r[2] += r[3] * L;
    r[4] -= O_SQR(p_norm) * L * (O_SQR(r[1] + O_SQR(r[2]))) / 2.0;
}

/* atpass.cpp:416-428 */
static void o_fastdrift(double* r, double NormL) {
    double dx = NormL * r[1];
    double dy = NormL * r[3];
    r[0] += dx;
    r[2] += dy;
    r[4] -= NormL * (r[1] * r[1] + r[3] * r[3]) / (2 * (1 + r[5]));
}

/* atpass.cpp:15-72 — linear thick quadrupole */
static void o_quad6(double* r, double L, double K) {
    double p_norm = 1 / (1 + r[5]);
    double x, xpr, y, ypr, g, t, lt;
    double M12, M21, M34, M43, MVD, MHD;
    if (K == 0) { o_drift(r, L); return; }
    x = r[0];
    xpr = r[1] * p_norm;
    y = r[2];
    ypr = r[3] * p_norm;
    g = fabs(K) / (1 + r[5]);
    t = sqrt(g);
    lt = L * t;
    if (K > 0) {
        MHD = cos(lt); M12 = sin(lt) / t; M21 = -M12 * g;
        MVD = cosh(lt); M34 = sinh(lt) / t; M43 = M34 * g;
    } else {
        MHD = cosh(lt); M12 = sinh(lt) / t; M21 = M12 * g;
        MVD = cos(lt); M34 = sin(lt) / t; M43 = -M34 * g;
    }
    r[0] = MHD * x + M12 * xpr;
    r[1] = (M21 * x + MHD * xpr) / p_norm;
    r[2] = MVD * y + M34 * ypr;
    r[3] = (M43 * y + MVD * ypr) / p_norm;
    r[4] -= g * (x * x * (L - MHD * M12) - y * y * (L - MVD * M34)) / 4;
    r[4] -= (xpr * xpr * (L + MHD * M12) + ypr * ypr * (L + MVD * M34)) / 4;
    r[4] -= (x * xpr * M12 * M21 + y * ypr * M34 * M43) / 2;
}

/* atpass.cpp:76-187 — linear sector bend with gradient (ByError = 0 from ABend::pass) */
static void o_bend6(double* r, double L, double b_angle, double grd, double ByError) {
    double M12, M21, M34, M43, MVD, MHD;
    double x, xpr, y, ypr, delta;
    double sqrtG1 = 0, sqrtG2, arg1 = 0, arg2;
    double Kx = b_angle / L;
    double p_norm = 1 / (1 + r[5]);
    double G1 = (Kx * Kx + grd) * p_norm;
    double G2 = -grd * p_norm;
    if (G1 == 0) { MHD = 1; M12 = L; M21 = 0; }
    else if (G1 > 0) {
        sqrtG1 = sqrt(G1); arg1 = L * sqrtG1;
        MHD = cos(arg1); M12 = sin(arg1) / sqrtG1; M21 = -sin(arg1) * sqrtG1;
    } else {
        sqrtG1 = sqrt(-G1); arg1 = L * sqrtG1;
        MHD = cosh(arg1); M12 = sinh(arg1) / sqrtG1; M21 = sinh(arg1) * sqrtG1;
    }
    if (G2 == 0) { MVD = 1; M34 = L; M43 = 0; }
    else if (G2 > 0) {
        sqrtG2 = sqrt(G2); arg2 = L * sqrtG2;
        MVD = cos(arg2); M34 = sin(arg2) / sqrtG2; M43 = -sin(arg2) * sqrtG2;
    } else {
        sqrtG2 = sqrt(-G2); arg2 = L * sqrtG2;
        MVD = cosh(arg2); M34 = sinh(arg2) / sqrtG2; M43 = sinh(arg2) * sqrtG2;
    }
    x = r[0];
    xpr = r[1] * p_norm;
    y = r[2];
    ypr = r[3] * p_norm;
    delta = r[5];
    r[0] = MHD * x + M12 * xpr;
    r[1] = (M21 * x + MHD * xpr) / p_norm;
    if (G1 == 0) {
        r[0] += (delta * p_norm - ByError) * L * L * Kx / 2;
        r[1] += (delta * p_norm - ByError) * L * Kx / p_norm;
    } else if (G1 > 0) {
        r[0] += (delta * p_norm - ByError) * (1 - cos(arg1)) * Kx / G1;
        r[1] += (delta * p_norm - ByError) * sin(arg1) * Kx / (sqrtG1 * p_norm);
    } else {
        r[0] += (delta * p_norm - ByError) * (1 - cosh(arg1)) * Kx / G1;
        r[1] += (delta * p_norm - ByError) * sinh(arg1) * Kx / (sqrtG1 * p_norm);
    }
    r[2] = MVD * y + M34 * ypr;
    r[3] = (M43 * y + MVD * ypr) / p_norm;
    r[4] -= xpr * xpr * (L + MHD * M12) / 4;
    if (G1 != 0) {
        r[4] -= (L - MHD * M12) * (x * x * G1 + (delta * p_norm - ByError) * (delta * p_norm - ByError) * Kx * Kx / G1
                                   - 2 * x * Kx * (delta * p_norm - ByError)) / 4;
        r[4] -= M12 * M21 * (x * xpr - xpr * (delta * p_norm - ByError) * Kx / G1) / 2;
        r[4] -= Kx * x * M12 + xpr * (1 - MHD) * Kx / G1 + (delta * p_norm - ByError) * (L - M12) * Kx * Kx / G1;
    }
    r[4] -= ((L - MVD * M34) * y * y * G2 + ypr * ypr * (L + MVD * M34)) / 4;
    r[4] -= M34 * M43 * y * ypr / 2;
}

/* atpass.cpp:190-196 — hard-edge fringe */
static void o_edge(double* r, double inv_rho, double edge_angle) {
    double psi = inv_rho * tan(edge_angle);
    r[1] += r[0] * psi;
    r[3] -= r[2] * psi;
}

/* atpass.cpp:199-235 — curved-frame multipole kick */
static void o_bndthinkick(double* r, const double* B, double L, double irho, int max_order) {
    double ReSum, ImSum = 0, ReSumTemp, K1, K2, h;
    int i;
    K1 = B[1];
    K2 = (max_order >= 2) ? B[2] : 0;
    h = irho;
    ReSum = B[max_order];
    for (i = max_order - 1; i >= 0; i--) {
        ReSumTemp = ReSum * r[0] - ImSum * r[2] + B[i];
        ImSum = ImSum * r[0] + ReSum * r[2];
        ReSum = ReSumTemp;
    }
    r[1] -= L * (-h * r[5] + ReSum + h * (h * r[0] + K1 * (r[0] * r[0] - 0.5 * r[2] * r[2]) + K2 * (r[0] * r[0] * r[0] - 4.0 / 3.0 * r[0] * r[2] * r[2])));
    r[3] += L * (ImSum + h * (K1 * r[0] * r[2] + 4.0 / 3.0 * K2 * r[0] * r[0] * r[2] + (h / 6.0 * K1 - K2 / 3.0) * r[2] * r[2] * r[2]));
    r[4] -= L * h * r[0];
}

/* atpass.cpp:237-253 */
static double o_B2perp(double bx, double by, double irho, double x, double xpr, double y, double ypr) {
    double v_norm2;
    (void)y;
    v_norm2 = 1 / (O_SQR(1 + x * irho) + O_SQR(xpr) + O_SQR(ypr));
    return ((O_SQR(by * (1 + x * irho)) + O_SQR(bx * (1 + x * irho)) + O_SQR(bx * ypr - by * xpr)) * v_norm2);
}

/* atpass.cpp:255-339 — kick with classical radiation (flag 1) or radiation + QE (flag 2) */
static void o_bndthinkickrad(double* r, const double* B, double L, double irho, double E0,
                             int max_order, int flag_rad, orc_rng* g) {
    double ReSum, ImSum = 0, ReSumTemp, K1, K2, h;
    double x, xpr, y, ypr, p_norm, B2P;
    double CRAD = O_CGAMMA * E0 * E0 * E0 / (O_TWOPI * 1e9);
    double uc_E0 = 0.665 * E0 * E0 / 1.0e6 / 2.99792458E8 * fabs(irho) * 1000;
    int i;
    K1 = B[1];
    K2 = (max_order >= 2) ? B[2] : 0;
    h = irho;
    ReSum = B[max_order];
    for (i = max_order - 1; i >= 0; i--) {
        ReSumTemp = ReSum * r[0] - ImSum * r[2] + B[i];
        ImSum = ImSum * r[0] + ReSum * r[2];
        ReSum = ReSumTemp;
    }
    p_norm = 1 / (1 + r[5]);
    x = r[0];
    xpr = r[1] * p_norm;
    y = r[2];
    ypr = r[3] * p_norm;
    ImSum += h * (K1 * h - K2) * y * y * y / 6.0;
    ReSum += -K1 * h * y * y / 2.0 + h * (K1 * h - K2) * x * y * y / 2.0;
    B2P = o_B2perp(ImSum, ReSum + irho, irho, x, xpr, y, ypr);
    if (flag_rad == 1) {
        r[5] = r[5] - CRAD * O_SQR(1 + r[5]) * B2P * (1 + x * irho + (O_SQR(xpr) + O_SQR(ypr)) / 2) * L;
    } else if (flag_rad == 2) {
        double mean_dpp = CRAD * O_SQR(1 + r[5]) * B2P * (1 + x * irho + (O_SQR(xpr) + O_SQR(ypr)) / 2) * L;
        double sigma_dpp;
        if (mean_dpp >= 0) sigma_dpp = sqrt(55 * sqrt(3) / 72.0 * uc_E0 * mean_dpp);
        else sigma_dpp = sqrt(-55 * sqrt(3) / 72.0 * uc_E0 * mean_dpp);
        double gr = g ? orc_gauss(g) : 0.0;
        r[5] = r[5] - (mean_dpp + gr * sigma_dpp);
    }
    p_norm = 1 / (1 + r[5]);
    r[1] = xpr / p_norm;
    r[3] = ypr / p_norm;
    r[1] -= L * (-h * r[5] + ReSum + h * (h * r[0] + K1 * (r[0] * r[0] - 0.5 * r[2] * r[2]) + K2 * (r[0] * r[0] * r[0] - 4.0 / 3.0 * r[0] * r[2] * r[2])));
    r[3] += L * (ImSum + h * (K1 * r[0] * r[2] + 4.0 / 3.0 * K2 * r[0] * r[0] * r[2] + (h / 6.0 * K1 - K2 / 3.0) * r[2] * r[2] * r[2]));
    r[4] -= L * h * r[0];
}

/* atpass.cpp:343-355 — the curved "hx" drift */
static void o_bendhxdrift(double* r, double L, double h) {
    double hs = h * L;
    double i1pd = 1.0 / (1 + r[5]);
    double x = r[0], px = r[1], py = r[3];
    r[0] += (1 + h * x) * px * i1pd * L + 1 / 4. * hs * L * (px * px - py * py) * i1pd * i1pd;
    r[1] -= hs * (px * px + py * py) * i1pd / 2.0;
    r[2] += (1.0 + h * x) * i1pd * py * L * (1. + px * hs / 2.0);
    r[4] -= (1.0 + h * x) * i1pd * i1pd * L / 2.0 * (px * px + py * py);
}

/* atpass.cpp:358-414 — straight multipole kick (complex Horner) */
static void o_strthinkick(double* r, const double* A, const double* B, double L, int max_order) {
    int i;
    double ReSum = B[max_order];
    double ImSum = A[max_order];
    double ReSumTemp;
    for (i = max_order - 1; i >= 0; i--) {
        ReSumTemp = ReSum * r[0] - ImSum * r[2] + B[i];
        ImSum = ImSum * r[0] + ReSum * r[2] + A[i];
        ReSum = ReSumTemp;
    }
    r[1] -= L * ReSum;
    r[3] += L * ImSum;
}

/* ------------------------------------------------------------------------------------------ */
/* Element passes (accel.cpp)                                                                   */
/* ------------------------------------------------------------------------------------------ */
static int o_aperture_test(double* r6, const double* f) {
    if (r6[0] <= f[0] || r6[0] >= f[1] || r6[2] <= f[2] || r6[2] >= f[3]) {
        r6[4] = (r6[0] <= f[0]) * 1 + (r6[0] >= f[1]) * 2 + (r6[2] <= f[2]) * 3 + (r6[2] >= f[3]) * 4;
        r6[0] = NAN;
        return 1;
    }
    return 0;
}

/* ATransWake::pass, accel.cpp:1603-1657: O(N^2) resonator sum over the particles it is given. */
static void o_transwake(const accel_elem_desc* e, double* r, int N) {
    double len = e->len, energy = e->f[0], Ne = e->f[1], Wx = e->f[2], fRx = e->f[3], Qx = e->f[4];
    double Wy = e->f[5], fRy = e->f[6], Qy = e->f[7];
    double q = Ne / N * 1000;
    double kRx = 2 * O_PI * fRx * 1.0e9 / O_C0;
    double kRy = 2 * O_PI * fRy * 1.0e9 / O_C0;
    double ax = kRx / 2 / Qx, ay = kRy / 2 / Qy;
    double kbarRx = kRx * sqrt(1.0 - 0.25 / O_SQR(Qx));
    double kbarRy = kRy * sqrt(1.0 - 0.25 / O_SQR(Qy));
    for (int i = 0; i < N; i++) {
        if (isnan(r[6 * i])) continue;
        double* r6 = r + 6 * i;
        if (len != 0) o_fastdrift(r6, 0.5 * len / (1 + r6[5]));
        if (e->flags) {
            double dxp = 0, dyp = 0;
            for (int j = 0; j < N; j++) {
                if (isnan(r[6 * j])) continue;
                if (i == j) continue;
                double* rj6 = r + 6 * j;
                double zij = r6[4] - rj6[4];
                if (zij > 0) continue;
                dxp = dxp - q * Wx * exp(ax * zij) * sin(kbarRx * zij) * rj6[0] / energy / 1.0e6;
                dyp = dyp - q * Wy * exp(ay * zij) * sin(kbarRy * zij) * rj6[2] / energy / 1.0e6;
            }
            r6[1] += dxp * (1 + r6[5]);
            r6[3] += dyp * (1 + r6[5]);
        }
        if (len != 0) o_fastdrift(r6, 0.5 * len / (1 + r6[5]));
    }
}

/* NEW — longitudinal broadband resonator wake, applied from a z histogram.
 *   W(s) = (w_r R_s / Q) e^{-a s/c} [cos(wb s/c) - (a/wb) sin(wb s/c)],  a = w_r/(2Q),
 *   wb = sqrt(w_r^2 - a^2), for a source a distance s >= 0 ahead (larger z leads, the convention
 *   of ATransWake's z_ij <= 0 test); W(0) enters with weight 1/2 (beam-loading theorem).
 * Binning: nbins bins over [zmin, zmax] of the live particles, nearest-grid-point deposit and
 * kick.  delta -= V / (E[MeV] * 1e6), with V = sum over bins k at or ahead of the particle's bin
 * j of q_k W((k - j) dz).  Bin charge q_k = Charge[nC] * 1e-9 * count_k / nlive. */
void orc_longwake_voltage(int nbins, double dz, const double* counts, double qper,
                          double Rs, double fr, double Q, double* V) {
    double wr = O_TWOPI * fr;
    double a = wr / (2 * Q);
    double wb = sqrt(wr * wr - a * a);
    double amp = wr * Rs / Q;
    for (int j = 0; j < nbins; j++) {
        double v = 0.5 * amp * counts[j] * qper;
        for (int k = j + 1; k < nbins; k++) {
            double tau = (k - j) * dz / O_C0;
            double w = amp * exp(-a * tau) * (cos(wb * tau) - (a / wb) * sin(wb * tau));
            v += w * counts[k] * qper;
        }
        V[j] = v;
    }
}

static void o_longwake(const accel_elem_desc* e, double* r, int N) {
    double len = e->len;
    int nbins = (int)e->f[5];
    if (nbins < 1) nbins = 1;
    if (nbins > 4096) nbins = 4096;
    for (int i = 0; i < N; i++)
        if (!isnan(r[6 * i]) && len != 0) o_fastdrift(r + 6 * i, 0.5 * len / (1 + r[6 * i + 5]));
    if (e->flags) {
        double zmin = INFINITY, zmax = -INFINITY;
        int nlive = 0;
        for (int i = 0; i < N; i++) {
            if (isnan(r[6 * i])) continue;
            double z = r[6 * i + 4];
            if (z < zmin) zmin = z;
            if (z > zmax) zmax = z;
            nlive++;
        }
        if (nlive > 0) {
            double dz = (zmax - zmin) / nbins;
            if (!(dz > 0)) dz = 1e-12;
            double inv_dz = 1.0 / dz;
            double* counts = (double*)calloc((size_t)nbins, sizeof(double));
            double* V = (double*)calloc((size_t)nbins, sizeof(double));
            for (int i = 0; i < N; i++) {
                if (isnan(r[6 * i])) continue;
                int b = (int)((r[6 * i + 4] - zmin) * inv_dz);
                if (b < 0) b = 0;
                if (b > nbins - 1) b = nbins - 1;
                counts[b] += 1.0;
            }
            double qper = e->f[1] * 1e-9 / nlive;
            orc_longwake_voltage(nbins, dz, counts, qper, e->f[2], e->f[3], e->f[4], V);
            double inv_e = 1.0 / (e->f[0] * 1e6);
            for (int i = 0; i < N; i++) {
                if (isnan(r[6 * i])) continue;
                int b = (int)((r[6 * i + 4] - zmin) * inv_dz);
                if (b < 0) b = 0;
                if (b > nbins - 1) b = nbins - 1;
                r[6 * i + 5] -= V[b] * inv_e;
            }
            free(counts);
            free(V);
        }
    }
    for (int i = 0; i < N; i++)
        if (!isnan(r[6 * i]) && len != 0) o_fastdrift(r + 6 * i, 0.5 * len / (1 + r[6 * i + 5]));
}

int orc_pass_element(const accel_elem_desc* e, double* r, int N, orc_rng* g) {
    const double len = e->len;
    switch (e->type) {
    case ACCEL_DRIFT: /* ADrift::pass accel.cpp:158-177 */
        for (int i = 0; i < N; i++) {
            if (isnan(r[6 * i])) continue;
            double* r6 = r + 6 * i;
            o_fastdrift(r6, len / (1.0 + r6[5]));
        }
        return 0;
    case ACCEL_QUAD: /* AQuad::pass accel.cpp:193-209 */
        for (int i = 0; i < N; i++) {
            if (isnan(r[6 * i])) continue;
            o_quad6(r + 6 * i, len, e->f[0]);
        }
        return 0;
    case ACCEL_CORRECTOR: /* ACorrector::pass accel.cpp:270-292 */
        for (int i = 0; i < N; i++) {
            if (isnan(r[6 * i])) continue;
            double* r6 = r + 6 * i;
            double pn = (1 + r6[5]);
            if (len != 0) o_fastdrift(r6, 0.5 * len / pn);
            r6[1] += e->f[0] / pn;
            r6[3] += e->f[1] / pn;
            if (len != 0) o_fastdrift(r6, 0.5 * len / pn);
        }
        return 0;
    case ACCEL_APERTURE: /* AAperture::pass accel.cpp:337-387 */
        for (int i = 0; i < N; i++) {
            if (isnan(r[6 * i])) continue;
            double* r6 = r + 6 * i;
            if (o_aperture_test(r6, e->f)) continue;
            if (len != 0) {
                o_fastdrift(r6, len / (1 + r6[5]));
                o_aperture_test(r6, e->f);
            }
        }
        return 0;
    case ACCEL_MONITOR: /* AMonitor::pass prints only; coordinates untouched */
        return 0;
    case ACCEL_BEND: { /* ABend::pass accel.cpp:523-550 */
        double irho = e->f[4];
        for (int i = 0; i < N; i++) {
            if (isnan(r[6 * i])) continue;
            double* r6 = r + 6 * i;
            o_edge(r6, irho, e->f[1]);
            o_bend6(r6, len, e->f[0], e->f[3], 0);
            o_edge(r6, irho, e->f[2]);
        }
        return 0;
    }
    case ACCEL_BENDMPOLE: { /* ABendMPole::pass accel.cpp:649-705 */
        double SL = len / e->nslice;
        double L1 = SL * O_DRIFT1, L2 = SL * O_DRIFT2, K1 = SL * O_KICK1, K2 = SL * O_KICK2;
        double irho = e->f[4], energy = e->f[3];
        int mo = e->max_npole - 1, rad = e->flags;
        const double* B = e->poly_b;
        if (mo < 0) return ACCEL_E_INVALID;
        for (int i = 0; i < N; i++) {
            if (isnan(r[6 * i])) continue;
            double* r6 = r + 6 * i;
            o_edge(r6, irho, e->f[1]);
            for (int m = 0; m < e->nslice; m++) {
                if (rad <= 1) {
                    o_bendhxdrift(r6, L1, irho);
                    if (rad) o_bndthinkickrad(r6, B, K1, irho, energy, mo, rad, g);
                    else o_bndthinkick(r6, B, K1, irho, mo);
                    o_bendhxdrift(r6, L2, irho);
                    if (rad) o_bndthinkickrad(r6, B, K2, irho, energy, mo, rad, g);
                    else o_bndthinkick(r6, B, K2, irho, mo);
                    o_bendhxdrift(r6, L2, irho);
                    if (rad) o_bndthinkickrad(r6, B, K1, irho, energy, mo, rad, g);
                    else o_bndthinkick(r6, B, K1, irho, mo);
                    o_bendhxdrift(r6, L1, irho);
                } else if (rad == 2) {
                    o_bendhxdrift(r6, 0.5 * SL, irho);
                    o_bndthinkickrad(r6, B, SL, irho, energy, mo, rad, g);
                    o_bendhxdrift(r6, 0.5 * SL, irho);
                }
            }
            o_edge(r6, irho, e->f[2]);
        }
        return 0;
    }
    case ACCEL_STRMPOLE: { /* AStrMPole::pass accel.cpp:800-847: Horner always at order 9 */
        double SL = len / e->nslice;
        double L1 = SL * O_DRIFT1, L2 = SL * O_DRIFT2, K1 = SL * O_KICK1, K2 = SL * O_KICK2;
        const double *A = e->poly_a, *B = e->poly_b;
        for (int i = 0; i < N; i++) {
            if (isnan(r[6 * i])) continue;
            double* r6 = r + 6 * i;
            if (len == 0) {
                o_strthinkick(r6, A, B, 1.0, ACCEL_MAX_MPOLE - 1);
            } else {
                for (int m = 0; m < e->nslice; m++) {
                    double norm = 1 / (1 + r6[5]);
                    double NormL1 = L1 * norm, NormL2 = L2 * norm;
                    o_fastdrift(r6, NormL1);
                    o_strthinkick(r6, A, B, K1, ACCEL_MAX_MPOLE - 1);
                    o_fastdrift(r6, NormL2);
                    o_strthinkick(r6, A, B, K2, ACCEL_MAX_MPOLE - 1);
                    o_fastdrift(r6, NormL2);
                    o_strthinkick(r6, A, B, K1, ACCEL_MAX_MPOLE - 1);
                    o_fastdrift(r6, NormL1);
                }
            }
        }
        return 0;
    }
    case ACCEL_CAVITY: { /* ACavity::pass accel.cpp:903-923 */
        double nv = e->f[0] / e->f[3];
        for (int i = 0; i < N; i++) {
            if (isnan(r[6 * i])) continue;
            double* r6 = r + 6 * i;
            if (len != 0) o_fastdrift(r6, 0.5 * len / (1 + r6[5]));
            if (e->flags) r6[5] += nv * sin(O_TWOPI * e->f[1] * r6[4] / O_C0 + e->f[2]);
            if (len != 0) o_fastdrift(r6, 0.5 * len / (1 + r6[5]));
        }
        return 0;
    }
    case ACCEL_TRANSWAKE:
        o_transwake(e, r, N);
        return 0;
    case ACCEL_LONGWAKE:
        o_longwake(e, r, N);
        return 0;
    case ACCEL_MATRIX: /* AMatrix::pass accel.cpp:1699-1730 */
        for (int i = 0; i < N; i++) {
            if (isnan(r[6 * i])) continue;
            double* r6 = r + 6 * i;
            double tr[6];
            if (len != 0) o_fastdrift(r6, 0.5 * len / (1 + r6[5]));
            for (int j = 0; j < 6; j++) {
                const double* m = e->mat + 6 * j;
                tr[j] = m[0] * r6[0] + m[1] * r6[1] + m[2] * r6[2] + m[3] * r6[3] + m[4] * r6[4] + m[5] * r6[5];
            }
            for (int j = 0; j < 6; j++) r6[j] = tr[j];
            if (len != 0) o_fastdrift(r6, 0.5 * len / (1 + r6[5]));
        }
        return 0;
    case ACCEL_SYNCRAD: { /* ASyncRad::pass accel.cpp:1806-1854; flags bit0 damping, bit1 QE */
        double energy = e->f[0], U0 = e->f[1], Jx = e->f[2], Jy = e->f[3];
        double Jz = 4 - Jx - Jy;
        double alfx = U0 / 2. / energy * Jx, alfy = U0 / 2. / energy * Jy, alfz = U0 / 2. / energy * Jz;
        double sx = sqrt(2. * alfx), sy = sqrt(2. * alfy), sz = sqrt(2. * alfz);
        double sigx = sqrt(e->f[4] * e->f[7]), sigy = sqrt(e->f[5] * e->f[8]);
        for (int i = 0; i < N; i++) {
            if (isnan(r[6 * i])) continue;
            double* r6 = r + 6 * i;
            if (len != 0) o_fastdrift(r6, 0.5 * len / (1 + r6[5]));
            if (e->flags & 1) {
                r6[0] *= (1 - alfx);
                r6[2] *= (1 - alfy);
                r6[5] *= (1 - alfz);
            }
            if ((e->flags & 2) && g) {
                r6[0] += sigx * sx * orc_gauss(g);
                r6[2] += sigy * sy * orc_gauss(g);
                r6[5] += e->f[6] * sz * orc_gauss(g);
            }
            if (len != 0) o_fastdrift(r6, 0.5 * len / (1 + r6[5]));
        }
        return 0;
    }
    default:
        return ACCEL_E_UNSUPPORTED;
    }
}

static int o_is_collective(int type) { return type == ACCEL_TRANSWAKE || type == ACCEL_LONGWAKE; }

/* ALine::pass(r, N, st, ed), aline.cpp:313-329: each thread takes a contiguous block of particles
 * through the elements.  Wake elements need the whole beam, so the line is split at them. */
int orc_pass_line(const accel_elem_desc* el, int n, double* r, int N, int st, int ed,
                  int nthreads, orc_rng* g) {
    if (st < 0 || ed > n || st > ed) return ACCEL_E_INVALID;
    int a = st;
    while (a < ed) {
        int b = a;
        while (b < ed && !o_is_collective(el[b].type)) b++;
        if (b > a) {
            int status = 0;
            if (nthreads > 1 && !g) {
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads) reduction(min : status)
                {
                    int t = omp_get_thread_num(), T = omp_get_num_threads();
                    int s0 = (int)((long long)t * N / T), s1 = (int)((long long)(t + 1) * N / T);
                    for (int k = a; k < b; k++) {
                        int st_k = orc_pass_element(el + k, r + 6 * (size_t)s0, s1 - s0, NULL);
                        if (st_k < status) status = st_k;
                    }
                }
#else
                for (int k = a; k < b; k++) { int s = orc_pass_element(el + k, r, N, g); if (s < status) status = s; }
#endif
            } else {
                for (int k = a; k < b; k++) { int s = orc_pass_element(el + k, r, N, g); if (s < status) status = s; }
            }
            if (status < 0) return status;
        }
        if (b < ed) {
            int s = orc_pass_element(el + b, r, N, g);
            if (s < 0) return s;
            b++;
        }
        a = b;
    }
    return 0;
}

int orc_track(const accel_elem_desc* el, int n, double* r, int N, int nturn, int32_t* loss_turn,
              int nthreads, uint64_t seed) {
    orc_rng g;
    orc_rng* gp = NULL;
    for (int k = 0; k < n; k++)
        if ((el[k].type == ACCEL_BENDMPOLE && el[k].flags == 2) || (el[k].type == ACCEL_SYNCRAD && (el[k].flags & 2)))
            gp = &g;
    if (gp) orc_rng_seed(gp, seed);
    if (loss_turn)
        for (int i = 0; i < N; i++) loss_turn[i] = -1;
    for (int t = 0; t < nturn; t++) {
        int s = orc_pass_line(el, n, r, N, 0, n, nthreads, gp);
        if (s < 0) return s;
        if (loss_turn)
            for (int i = 0; i < N; i++)
                if (loss_turn[i] < 0 && isnan(r[6 * i])) loss_turn[i] = t;
    }
    return 0;
}

/* ALine::getm66, aline.cpp:900-927: 12 particles at +/-delta on each axis, elements passed
 * directly (no OpenMP), m[i][j] = (r+ - r-) / 2 / delta. */
void orc_m66(const accel_elem_desc* el, int n, int st, int ed, double dpp, double delta, double* m36) {
    double r0[6] = {0, 0, 0, 0, 0, 0};
    r0[5] = dpp;
    /* the reference adds dpp after placing +/-delta: r[5] = (+/-delta or 0) + dpp */
    double r[72];
    for (int i = 0; i < 72; i++) r[i] = 0.0;
    r[0] = r[7] = r[14] = r[21] = r[28] = r[35] = delta;
    r[36 + 0] = r[36 + 7] = r[36 + 14] = r[36 + 21] = r[36 + 28] = r[36 + 35] = -delta;
    for (int i = 0; i < 12; i++) r[i * 6 + 5] += dpp;
    (void)r0;
    for (int k = st; k < ed; k++) orc_pass_element(el + k, r, 12, NULL);
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) m36[6 * i + j] = (r[j * 6 + i] - r[j * 6 + i + 36]) / 2.0 / delta;
}

void orc_m66_at(const accel_elem_desc* el, int n, int st, int ed, const double* p, double delta, double* m36) {
    double r[72];
    (void)n;
    for (int j = 0; j < 12; j++)
        for (int k = 0; k < 6; k++) r[6 * j + k] = p[k];
    for (int j = 0; j < 6; j++) { r[6 * j + j] += delta; r[36 + 6 * j + j] -= delta; }
    for (int k = st; k < ed; k++) orc_pass_element(el + k, r, 12, NULL);
    for (int i = 0; i < 6; i++)
        for (int j = 0; j < 6; j++) m36[6 * i + j] = (r[j * 6 + i] - r[j * 6 + i + 36]) / 2.0 / delta;
}

/* calc_beam_stat, utility.cpp:387-438 */
int orc_beam_stat(const double* r, int N, double* ar, double* sigr, double* sigrr) {
    int nlive = 0;
    for (int i = 0; i < 6; i++) { ar[i] = 0; sigr[i] = 0; }
    for (int j = 0; j < N; j++) {
        const double* pr = r + 6 * j;
        if (isnan(pr[0])) continue;
        nlive++;
        for (int i = 0; i < 6; i++) ar[i] += pr[i];
    }
    for (int i = 0; i < 6; i++) ar[i] /= nlive;
    for (int j = 0; j < N; j++) {
        const double* pr = r + 6 * j;
        if (isnan(pr[0])) continue;
        for (int i = 0; i < 6; i++) sigr[i] += O_SQR(pr[i] - ar[i]);
    }
    for (int i = 0; i < 6; i++) { sigr[i] /= nlive; sigr[i] = sqrt(sigr[i]); }
    if (sigrr) {
        for (int i = 0; i < 6; i++) sigrr[i] = 0;
        for (int j = 0; j < N; j++) {
            const double* pr = r + 6 * j;
            if (isnan(pr[0])) continue;
            sigrr[0] += (pr[0] - ar[0]) * (pr[1] - ar[1]);
            sigrr[1] += (pr[2] - ar[2]) * (pr[3] - ar[3]);
            sigrr[2] += (pr[0] - ar[0]) * (pr[5] - ar[5]);
            sigrr[3] += (pr[1] - ar[1]) * (pr[5] - ar[5]);
            sigrr[4] += (pr[2] - ar[2]) * (pr[4] - ar[4]);
            sigrr[5] += (pr[3] - ar[3]) * (pr[4] - ar[4]);
        }
        for (int i = 0; i < 6; i++) sigrr[i] /= nlive;
    }
    return nlive;
}

/* ALine::set_rad_onoff / set_cavity_onoff / set_wake_onoff (aline.cpp:258-293, 429-463) */
void orc_set_flags(accel_elem_desc* el, int n, int rad_flag, int cavity_on, int wake_on) {
    for (int k = 0; k < n; k++) {
        accel_elem_desc* e = el + k;
        if (e->type == ACCEL_BENDMPOLE) e->flags = (rad_flag <= 2 && rad_flag >= 0) ? rad_flag : 0;
        else if (e->type == ACCEL_SYNCRAD) {
            if (rad_flag == ACCEL_RAD_LUMP) e->flags = 3;
            else if (rad_flag == ACCEL_RAD_LUMP_DAMP) e->flags = 1;
            else if (rad_flag == ACCEL_RAD_LUMP_QE) e->flags = 2;
            else e->flags = 0;
        } else if (e->type == ACCEL_CAVITY) {
            if (cavity_on >= 0) e->flags = cavity_on ? 1 : 0;
        } else if (e->type == ACCEL_TRANSWAKE || e->type == ACCEL_LONGWAKE) {
            if (wake_on >= 0) e->flags = wake_on ? 1 : 0;
        }
    }
}
