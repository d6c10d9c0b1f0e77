// Oracle (test infrastructure only): thermal-balance restatement.  See
// orc_thermal.h.
#include "orc_thermal.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace orc {

// ---- gaunt.f90:18-156 -----------------------------------------------------
// The Fortran declares the working variables REAL (single precision) and
// the 88 expansion coefficients REAL(8); mixed expressions promote to
// double and round back on assignment.  Restated with float/double to keep
// the same rounding sequence.
static const double kHummerD[88] = {
    8.986940175e+00, -4.009515855e+00, 8.808871266e-01, 2.640245111e-02, -4.580645915e-02, -3.568055702e-03,
    2.827798067e-03, 3.365860195e-04, -8.006936989e-01, 9.466021705e-01, 9.043402532e-02, -9.608451450e-02,
    -1.885629865e-02, 1.050313890e-02, 2.800889961e-03, -1.078209202e-03, -3.781305103e-01, 1.102726332e-01,
    -1.543619180e-02, 8.310561114e-03, 2.179620525e-02, 4.259726289e-03, -4.181588794e-03, -1.770208330e-03,
    1.877213132e-02, -1.004885705e-01, -5.483366378e-02, -4.520154409e-03, 8.366530426e-03, 3.700273930e-03,
    6.889320423e-04, 9.460313195e-05, 7.300158392e-02, 3.576785497e-03, -4.545307025e-03, -1.017965604e-02,
    -9.530211924e-03, -3.450186162e-03, 1.040482914e-03, 1.407073544e-03, -1.744671550e-03, 2.864013856e-02,
    1.903394837e-02, 7.091074494e-03, -9.668371391e-04, -2.999107465e-03, -1.820642230e-03, -3.874082085e-04,
    -1.707268366e-02, -4.694254776e-03, 1.311691517e-03, 5.316703136e-03, 5.178193095e-03, 2.451228935e-03,
    -2.277321615e-05, -8.182359057e-04, 2.567331664e-04, -9.155339970e-03, -6.997479192e-03, -3.571518641e-03,
    -2.096101038e-04, 1.553822487e-03, 1.509584686e-03, 6.212627837e-04, 4.098322531e-03, 1.635218463e-03,
    -5.918883504e-04, -2.333091048e-03, -2.484138313e-03, -1.359996060e-03, -5.371426147e-05, 5.553549563e-04,
    3.837562402e-05, 2.938325230e-03, 2.393747064e-03, 1.328839809e-03, 9.135013312e-05, -7.137252303e-04,
    -7.656848158e-04, -3.504683798e-04, -8.491991820e-04, -3.615327726e-04, 3.148015257e-04, 8.909207650e-04,
    9.869737522e-04, 6.134671184e-04, 1.068883394e-04, -2.046080100e-04};

void get_gaunt_ff(float z, float log10Te, const float* xlf, int n, float* g) {
    // d(j, k) column-major: dd((k-1)*8 + j)
    auto d = [](int j, int k) { return kHummerD[(k - 1) * 8 + (j - 1)]; };
    float b[12], c[9];
    float xlrkt;
    if (log10Te < 2.5f) xlrkt = 5.1983649f - 2.5f;
    else if (log10Te > 8.f) xlrkt = 5.1983649f - 8.f;
    else xlrkt = 5.1983649f - log10Te;
    const float txg = 0.66666667f * (2.0f * z + xlrkt);
    const float gamma2 = powf(10.0f, txg * 1.5f);
    const float con = 0.72727273f * xlrkt + 0.90909091f;
    for (int j = 1; j <= 8; ++j) {
        int ir = 9;
        b[11] = (float)d(j, 11);
        b[10] = (float)((double)(txg * b[11]) + d(j, 10));
        for (int i = 1; i <= 9; ++i) {
            b[ir] = (float)((double)(txg * b[ir + 1] - b[ir + 2]) + d(j, ir));
            ir = ir - 1;
        }
        c[j] = 0.25f * (b[1] - b[3]);
    }
    for (int i = 0; i < n; ++i) {
        const float txu = 0.72727273f * xlf[i] + con;
        const float u = powf(10.0f, (txu - .90909091f) / .72727273f);
        if (std::fabs(txu) <= 2.0f) {
            int ir = 6;
            b[8] = c[8];
            b[7] = txu * b[8] + c[7];
            for (int j = 1; j <= 6; ++j) {
                b[ir] = txu * b[ir + 1] - b[ir + 2] + c[ir];
                ir = ir - 1;
            }
            g[i] = b[1] - b[3];
        } else if (log10f(u) < -4.0f && gamma2 < 0.3f) {
            g[i] = 0.551329f * logf(2.24593f / u);
        } else if (log10f(u) < -4.0f && gamma2 >= 0.3f) {
            g[i] = 0.551329f * logf(0.944931f / u / sqrtf(gamma2));
        } else if (txu > 2.0f) {
            if (log10f(gamma2) < -3.f) {
                g[i] = sqrtf(0.9549297f / u);
            } else if (log10f(gamma2) < 0.0f) {
                const float slope = (sqrtf(12 * gamma2 / u) - sqrtf(0.9549297f / u)) / 3.0f;
                g[i] = sqrtf(12 * gamma2 / u) + slope * log10f(gamma2);
            } else {
                g[i] = sqrtf(12.f * gamma2 / u);
                g[i] = std::fmin(1.05f, g[i]);
            }
        }
    }
}

// gaunt_ff_mean, cooling_mod.f90:182-220 (64-point log-u midpoint grid).
double gaunt_ff_mean(double T, double Zc) {
    const int NU = 64;
    double u[NU], du[NU];
    float xlf[NU], g[NU];
    const double lo = std::log(1.0e-4), hi = std::log(20.0);
    for (int i = 1; i <= NU; ++i) {
        u[i - 1] = std::exp(lo + (hi - lo) * ((double)i - 0.5) / (double)NU);
        du[i - 1] = u[i - 1] * (hi - lo) / (double)NU;
    }
    const double ryd_over_kt = 13.605693 * EV2ERG / (KBOLTZ_CGS * T);
    for (int i = 0; i < NU; ++i) xlf[i] = (float)std::log10(u[i] / ryd_over_kt);
    for (int i = 0; i < NU; ++i) g[i] = 0.0f;
    get_gaunt_ff((float)std::log10(Zc), (float)std::log10(T), xlf, NU, g);
    double gm = 0.0;
    for (int i = 0; i < NU; ++i) gm = gm + (double)g[i] * std::exp(-u[i]) * du[i];
    return gm / (std::exp(-1.0e-4) - std::exp(-20.0));
}

void GffTable::build() {
    for (int i = 1; i <= 41; ++i) {
        logT[i - 1] = 2.0 + 4.0 * (double)(i - 1) / (double)(41 - 1);
        for (int iz = 1; iz <= 4; ++iz) z[i - 1][iz - 1] = gaunt_ff_mean(std::pow(10.0, logT[i - 1]), (double)iz);
    }
}

double GffTable::gbar(double T, int Z) const {
    const int iz = std::max(1, std::min(Z, 4));
    const double lt = std::min(std::max(std::log10(T), logT[0]), logT[40]);
    const int i = std::min((int)((lt - logT[0]) / (logT[1] - logT[0])) + 1, 41 - 1);
    const double w = (lt - logT[i - 1]) / (logT[i] - logT[i - 1]);
    return z[i - 1][iz - 1] * (1.0 - w) + z[i][iz - 1] * w;
}

// ---- cooling fits, cooling_mod.f90:98-134 ----------------------------------
bool CoolingFit::load(const std::string& path) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    int n = -1;
    while (std::getline(f, line)) {
        size_t a = line.find_first_not_of(" \t");
        if (a == std::string::npos || line[a] == '#') continue;
        n = std::atoi(line.c_str() + a);
        break;
    }
    if (n < 1) return false;
    A.resize(n);
    Ti.resize(n);
    for (int i = 0; i < n; ++i)
        if (!(f >> A[i] >> Ti[i])) return false;
    return true;
}

double CoolingFit::eval(double T) const {
    double lam = 0.0;
    for (size_t i = 0; i < A.size(); ++i) lam = lam + A[i] * std::exp(-Ti[i] / T);
    return lam / std::sqrt(T);
}

// ---- nlevel_mod.f90 -----------------------------------------------------------
bool NlevelAtom::load(const std::string& path) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
        size_t a = line.find_first_not_of(" \t");
        if (a == std::string::npos || line[a] == '#') continue;
        std::istringstream ss(line);
        std::string key;
        int n;
        ss >> key >> n;
        if (key == "NLEV") {
            nlev = n;
            for (int k = 0; k < n; ++k) {
                int idx;
                f >> idx >> g[k] >> e_cm1[k];
            }
            std::getline(f, line);
        } else if (key == "NRAD") {
            nrad = n;
            rl.resize(n); ru.resize(n); A.resize(n);
            for (int k = 0; k < n; ++k) f >> rl[k] >> ru[k] >> A[k];
            std::getline(f, line);
        } else if (key == "NUPS") {
            nups = n;
            ul_l.resize(n); ul_u.resize(n); ttype.resize(n); cups.resize(n); dery.resize(n);
            st_lo.resize(n); st_hi.resize(n); logf.resize(n); nc.resize(n); coef.assign(n, {});
            for (int k = 0; k < n; ++k) {
                std::getline(f, line);
                std::istringstream ls(line);
                ls >> ul_l[k] >> ul_u[k] >> ttype[k] >> cups[k] >> dery[k] >> st_lo[k] >> st_hi[k] >> logf[k] >> nc[k];
                coef[k].resize(nc[k]);
                for (int j = 0; j < nc[k]; ++j) ls >> coef[k][j];
            }
        }
    }
    return nlev > 0 && nups > 0;
}

static const double COLL_PREF = 8.629e-6;
static const double KB_OVER_RY = KBOLTZ_CGS / 2.1798723611035e-11;
static const double HC_ERG_CM = 1.9864458571489287e-16;

double NlevelAtom::ups(int k, double T) const {   // nlevel_mod.f90:119-152
    const double et = KB_OVER_RY * T / dery[k];
    double st;
    if (ttype[k] == 1 || ttype[k] == 4) st = 1.0 - std::log(cups[k]) / std::log(et + cups[k]);
    else st = et / (et + cups[k]);
    st = std::min(std::max(st, st_lo[k]), st_hi[k]);
    const double u = st_hi[k] > st_lo[k] ? 2.0 * (st - st_lo[k]) / (st_hi[k] - st_lo[k]) - 1.0 : 0.0;
    double b0 = 0.0, b1 = 0.0, b2;
    for (int j = nc[k]; j >= 2; --j) {
        b2 = b1;
        b1 = b0;
        b0 = 2.0 * u * b1 - b2 + coef[k][j - 1];
    }
    double y = u * b0 - b1 + coef[k][0];
    if (logf[k] == 1) y = std::pow(10.0, y);
    double r;
    switch (ttype[k]) {
        case 1: r = y * std::log(et + std::exp(1.0)); break;
        case 2: r = y; break;
        case 3: r = y / (et + 1.0); break;
        case 4: r = y * std::log(et + cups[k]); break;
        case 5: r = y / et; break;
        default: r = std::pow(10.0, y); break;
    }
    return std::max(r, 0.0);
}

// emitting_level (nlevel_mod.f90:168-181): orient a pair by energy.
static void emitting_level(const NlevelAtom& a, int i1, int i2, int& lo, int& hi, double& de) {
    if (a.e_cm1[i2 - 1] >= a.e_cm1[i1 - 1]) { lo = i1; hi = i2; } else { lo = i2; hi = i1; }
    de = (a.e_cm1[hi - 1] - a.e_cm1[lo - 1]) * HC_ERG_CM;
}

// nlevel_cooling_prepT (:247-271) + nlevel_cooling_solve (:274-326).
static void prepT(const NlevelAtom& a, double T, std::vector<double>& Rc, std::vector<double>& Rr) {
    const int M = NL_MAXLEV;
    Rc.assign(M * M, 0.0);
    Rr.assign(M * M, 0.0);
    for (int k = 0; k < a.nups; ++k) {
        int l, u;
        double de;
        emitting_level(a, a.ul_l[k], a.ul_u[k], l, u, de);
        const double ups = a.ups(k, T);
        const double q_ul = COLL_PREF / (a.g[u - 1] * std::sqrt(T)) * ups;
        const double q_lu = (a.g[u - 1] / a.g[l - 1]) * q_ul * std::exp(-de / (KBOLTZ_CGS * T));
        Rc[(u - 1) * M + (l - 1)] += q_lu;
        Rc[(l - 1) * M + (u - 1)] += q_ul;
    }
    for (int k = 0; k < a.nrad; ++k) {
        int l, u;
        double de;
        emitting_level(a, a.rl[k], a.ru[k], l, u, de);
        Rr[(l - 1) * M + (u - 1)] += a.A[k];
    }
}

static double solve(const NlevelAtom& a, const std::vector<double>& Rc, const std::vector<double>& Rr, double ne) {
    const int M = NL_MAXLEV, n = a.nlev;
    std::vector<double> R(M * M), Mx((size_t)M * (M + 1), 0.0), pop(M);
    for (int i = 0; i < M * M; ++i) R[i] = ne * Rc[i] + Rr[i];
    auto m = [&](int i, int j) -> double& { return Mx[(size_t)(i - 1) * (M + 1) + (j - 1)]; };
    for (int i = 1; i <= n; ++i)
        for (int j = 1; j <= n; ++j)
            if (i != j) {
                m(i, j) = R[(i - 1) * M + (j - 1)];
                m(i, i) = m(i, i) - R[(j - 1) * M + (i - 1)];
            }
    for (int j = 1; j <= n; ++j) m(1, j) = 1.0;
    m(1, n + 1) = 1.0;
    for (int i = 1; i <= n - 1; ++i) {
        int ip = i;
        for (int j = i + 1; j <= n; ++j)
            if (std::fabs(m(j, i)) > std::fabs(m(ip, i))) ip = j;
        if (ip != i)
            for (int j = i; j <= n + 1; ++j) std::swap(m(i, j), m(ip, j));
        for (int j = i + 1; j <= n; ++j) {
            const double fac = m(j, i) / m(i, i);
            for (int k = i; k <= n + 1; ++k) m(j, k) = m(j, k) - fac * m(i, k);
        }
    }
    for (int i = n; i >= 1; --i) {
        pop[i - 1] = m(i, n + 1);
        for (int j = i + 1; j <= n; ++j) pop[i - 1] = pop[i - 1] - m(i, j) * pop[j - 1];
        pop[i - 1] = pop[i - 1] / m(i, i);
    }
    double lam = 0.0;
    for (int k = 0; k < a.nrad; ++k) {
        int lo, hi;
        double de;
        emitting_level(a, a.rl[k], a.ru[k], lo, hi, de);
        lam = lam + pop[hi - 1] * a.A[k] * de;
    }
    return lam / ne;
}

double nlevel_cooling_at(const NlevelAtom& atom, double T, double ne) {
    std::vector<double> Rc, Rr;
    prepT(atom, T, Rc, Rr);
    return solve(atom, Rc, Rr, ne);
}

// ---- nlevel_cooling_mod.f90 ---------------------------------------------------
static double gT(int i) { return 2.0 + 0.01 * (double)(i - 1); }    // :90-95 (1-based)
static double gne(int j) { return -6.0 + 0.1 * (double)(j - 1); }

bool NlevelTable::build(const NlevelAtom& atom) {
    std::vector<double> lam((size_t)NT * NNE);
#pragma omp parallel for schedule(dynamic)
    for (int i = 1; i <= NT; ++i) {
        std::vector<double> Rc, Rr;
        prepT(atom, std::pow(10.0, gT(i)), Rc, Rr);
        for (int j = 1; j <= NNE; ++j) lam[(size_t)(i - 1) * NNE + (j - 1)] = solve(atom, Rc, Rr, std::pow(10.0, gne(j)));
    }
    lamref.resize(NT);
    Ssup.resize((size_t)NT * NNE);
    for (int i = 0; i < NT; ++i) lamref[i] = lam[(size_t)i * NNE];
    for (int i = 0; i < NT; ++i)
        for (int j = 0; j < NNE; ++j) Ssup[(size_t)i * NNE + j] = lam[(size_t)i * NNE + j] / std::max(lam[(size_t)i * NNE], TINEST);
    return true;
}

double NlevelTable::col(int it, int j, double w1, double wt) const {   // 1-based it, j
    const double Li = lamref[it - 1] * Ssup[(size_t)(it - 1) * NNE + (j - 1)];
    const double Lip = lamref[it] * Ssup[(size_t)it * NNE + (j - 1)];
    if (Li > 0.0 && Lip > 0.0) return std::exp(std::log(Li) + w1 * (std::log(Lip) - std::log(Li)));
    return Li * (1.0 - wt) + Lip * wt;
}

static void t_weights(double T, int& it, double& w1, double& wt) {
    const double lt = std::min(std::max(std::log10(T), gT(1)), gT(NlevelTable::NT));
    it = std::min((int)((lt - gT(1)) / 0.01) + 1, NlevelTable::NT - 1);
    w1 = (1.0 / std::pow(10.0, lt) - 1.0 / std::pow(10.0, gT(it))) / (1.0 / std::pow(10.0, gT(it + 1)) - 1.0 / std::pow(10.0, gT(it)));
    wt = std::min(std::max((lt - gT(it)) / (gT(it + 1) - gT(it)), 0.0), 1.0);
}

double NlevelTable::coeff(double T, double ne) const {
    int it;
    double w1, wt;
    t_weights(T, it, w1, wt);
    const double lne = std::log10(ne);
    if (lne <= gne(1)) return col(it, 1, w1, wt);
    if (lne >= gne(NNE)) return col(it, NNE, w1, wt);
    const int je = std::min((int)((lne - gne(1)) / 0.1) + 1, NNE - 1);
    const double wn = (lne - gne(je)) / (gne(je + 1) - gne(je));
    const double L0 = col(it, je, w1, wt), L1 = col(it, je + 1, w1, wt);
    if (L0 > 0.0 && L1 > 0.0) return std::exp(std::log(L0) + wn * (std::log(L1) - std::log(L0)));
    return L0 * (1.0 - wn) + L1 * wn;
}

double NlevelTable::low_density(double T) const {
    int it;
    double w1, wt;
    t_weights(T, it, w1, wt);
    return col(it, 1, w1, wt);
}

double NlevelTable::apply(double lam_fit, double T, double ne) const {
    const double lamref_ = low_density(T);
    const double S = coeff(T, ne) / std::max(lamref_, TINEST);
    const double fcov = std::min(1.0, lamref_ / std::max(lam_fit, TINEST));
    return lam_fit * (fcov * S + (1.0 - fcov));
}

bool Thermal::setup(const Par& p, std::string* err) {
    gff.build();
    std::string dir = p.atomic_dir;
    if (dir.empty()) dir = p.data_dir.empty() ? std::string("data/atomic") : p.data_dir + "/atomic";
    if (!hi_fit.load(dir + "/cooling_h_1.txt")) {
        if (err) *err = "cannot open " + dir + "/cooling_h_1.txt";
        return false;
    }
    use_hi_table = p.cooling_model == "local_ne";
    if (use_hi_table) {
        NlevelAtom atom;
        if (atom.load(dir + "/nlevel_h_1.txt")) hi_table.build(atom);
        else use_hi_table = false;   // no table: the fit value is used unchanged
    }
    return true;
}

// betaA/B_HII, beta_HeII/HeIII (cooling_mod.f90:139-175).
static double betaA_HII(double T) {
    const double lam = 2.0 * 157807.0 / T;
    return 1.778e-29 * T * std::pow(lam, 1.965) / std::pow(1.0 + std::pow(lam / 0.541, 0.502), 2.697);
}
static double betaB_HII(double T) {
    const double lam = 2.0 * 157807.0 / T;
    return 3.435e-30 * T * std::pow(lam, 1.970) / std::pow(1.0 + std::pow(lam / 2.250, 0.376), 3.720);
}
static double beta_HeIII(double T, bool caseA) {
    const double lam = 2.0 * 631515.0 / T;
    if (caseA) return 2.0 * 1.778e-29 * T * std::pow(lam, 1.965) / std::pow(1.0 + std::pow(lam / 0.541, 0.502), 2.697);
    return 2.0 * 3.435e-30 * T * std::pow(lam, 1.970) / std::pow(1.0 + std::pow(lam / 2.250, 0.376), 3.720);
}

double cooling_total(const Thermal& th, const RateModel& rm, bool caseA, double yHe, double T, double nH,
                     double ne, double xHI, double xHeI, double xHeII) {
    const double xHeIII = std::max(0.0, 1.0 - xHeI - xHeII);
    const double nHI = nH * xHI, nHII = nH * (1.0 - xHI);
    const double nHeI = nH * yHe * xHeI, nHeII = nH * yHe * xHeII, nHeIII = nH * yHe * xHeIII;
    double cool;
    const double bHeII = KBOLTZ_CGS * T * (caseA ? alphaA_HeII(rm, T) : alphaB_HeII(rm, T));
    if (caseA) cool = ne * (nHII * betaA_HII(T) + nHeII * bHeII + nHeIII * beta_HeIII(T, true));
    else cool = ne * (nHII * betaB_HII(T) + nHeII * bHeII + nHeIII * beta_HeIII(T, false));
    cool = cool + 1.42554e-27 * std::sqrt(T) * ne * ((nHII + nHeII) * th.gff.gbar(T, 1) + 4.0 * nHeIII * th.gff.gbar(T, 2));
    cool = cool + ne * (nHI * ci_HI(rm, T) * ETH_HI + nHeI * ci_HeI(rm, T) * ETH_HEI + nHeII * ci_HeII(rm, T) * ETH_HEII) * EV2ERG;
    const double fit = th.hi_fit.eval(T);
    const double lam = th.use_hi_table ? th.hi_table.apply(fit, T, ne) : fit;
    cool = cool + ne * nHI * lam;
    return cool;
}

}  // namespace orc

namespace orc {

namespace {

struct Bins1D {
    std::vector<double> ec, lum, sH, sHe1, sHe2;
};

// band_bins (check_g2a.py:94-103): geometric bin centres of nnu log-spaced
// bins, the Planck photon-energy shape integrated with 32 midpoint samples
// per bin, normalised to the band luminosity.
Bins1D band_bins_1d(const Sphere1D& s) {
    Bins1D b;
    const int n = s.nnu;
    std::vector<double> edge(n + 1);
    for (int i = 0; i <= n; ++i)
        edge[i] = std::exp(std::log(s.emin) + (std::log(s.emax) - std::log(s.emin)) * (double)i / (double)n);
    double tot = 0.0;
    for (int i = 0; i < n; ++i) {
        b.ec.push_back(std::sqrt(edge[i] * edge[i + 1]));
        const double w = edge[i + 1] - edge[i];
        double acc = 0.0;
        for (int k = 0; k < 32; ++k) {
            const double e = edge[i] + w * ((double)k + 0.5) / 32.0;
            acc += e * e * e / std::expm1(e * EV2ERG / (KBOLTZ_CGS * s.tstar));
        }
        b.lum.push_back(acc * w / 32.0);
        tot += b.lum.back();
    }
    for (int i = 0; i < n; ++i) {
        b.lum[i] *= s.lband / tot;
        b.sH.push_back(sigma_HI(b.ec[i]));
        b.sHe1.push_back(sigma_HeI(b.ec[i]));
        b.sHe2.push_back(sigma_HeII(b.ec[i]));
    }
    return b;
}

struct Rates1D {
    double gH, gHe1, gHe2, hH, hHe1, hHe2;
};

// net_rate (check_g2a.py:144-147): the ionization solved at T from the
// shell's state xs, heating from the attenuated fluxes minus cooling_total.
double net_1d(const Thermal& th, const RateModel& rm, const Sphere1D& s, const Rates1D& q, double T,
              const double xs[3], double out[3]) {
    double xHI = xs[0], xHeI = xs[1], xHeII = xs[2], ne = 0.0;
    solve_ion_cell(rm, s.yHe, q.gH, q.gHe1, q.gHe2, s.nH, T, false, xHI, xHeI, xHeII, ne);
    out[0] = xHI; out[1] = xHeI; out[2] = xHeII;
    const double heat = s.nH * (xHI * q.hH + s.yHe * (xHeI * q.hHe1 + xHeII * q.hHe2));
    return heat - cooling_total(th, rm, false, s.yHe, T, s.nH, ne, xHI, xHeI, xHeII);
}

}  // namespace

// reference_1d, check_g2a.py:150-207.
int thermal_1d(const Thermal& th, const RateModel& rm, const Sphere1D& s, int nr, int nsweep, double* r_pc,
               double* xHI, double* xHeI, double* xHeII, double* Te) {
    if (nr < 1 || nsweep < 1 || s.nnu < 1) return 1;
    const Bins1D b = band_bins_1d(s);
    const int nb = s.nnu;
    const double dr_pc = s.rsph_pc / (double)nr, dr_cm = dr_pc * PC2CM;
    for (int i = 0; i < nr; ++i) {
        r_pc[i] = ((double)i + 0.5) * dr_pc;
        xHI[i] = 1.0e-3; xHeI[i] = 0.0; xHeII[i] = 1.0; Te[i] = 1.0e4;
    }
    std::vector<double> prev(nr), tau(nb), flux(nb);
    for (int sweep = 0; sweep < nsweep; ++sweep) {
        std::copy(Te, Te + nr, prev.begin());
        std::fill(tau.begin(), tau.end(), 0.0);
        for (int i = 0; i < nr; ++i) {
            double xs[3] = {xHI[i], xHeI[i], xHeII[i]}, te = Te[i];
            const double rc = r_pc[i] * PC2CM;
            for (int pass = 0; pass < 2; ++pass) {
                Rates1D q = {0, 0, 0, 0, 0, 0};
                for (int k = 0; k < nb; ++k) {
                    const double kap = s.nH * (xs[0] * b.sH[k] + s.yHe * (xs[1] * b.sHe1[k] + xs[2] * b.sHe2[k]));
                    const double f = b.lum[k] * std::exp(-(tau[k] + 0.5 * kap * dr_cm)) / (4.0 * PI * rc * rc);
                    const double hnu = b.ec[k] * EV2ERG;
                    q.gH += f * b.sH[k] / hnu;
                    q.gHe1 += f * b.sHe1[k] / hnu;
                    q.gHe2 += f * b.sHe2[k] / hnu;
                    q.hH += f * b.sH[k] * (1.0 - ETH_HI / b.ec[k]);
                    q.hHe1 += f * b.sHe1[k] * (1.0 - ETH_HEI / b.ec[k]);
                    q.hHe2 += f * b.sHe2[k] * (1.0 - ETH_HEII / b.ec[k]);
                }
                double tlo = s.te_min, thi = s.te_max, xlo[3], xhi[3], xm[3];
                const double nlo = net_1d(th, rm, s, q, tlo, xs, xlo);
                const double nhi = net_1d(th, rm, s, q, thi, xs, xhi);
                if (nlo <= 0.0) {
                    te = tlo;
                    std::copy(xlo, xlo + 3, xs);
                } else if (nhi >= 0.0) {
                    te = thi;
                    std::copy(xhi, xhi + 3, xs);
                } else {
                    for (int it = 0; it < 60; ++it) {
                        const double tm = std::sqrt(tlo * thi);
                        if (net_1d(th, rm, s, q, tm, xs, xm) > 0.0) tlo = tm;
                        else thi = tm;
                        if (thi / tlo - 1.0 < 1.0e-5) break;
                    }
                    te = std::sqrt(tlo * thi);
                    net_1d(th, rm, s, q, te, xs, xm);
                    std::copy(xm, xm + 3, xs);
                }
            }
            xHI[i] = xs[0]; xHeI[i] = xs[1]; xHeII[i] = xs[2]; Te[i] = te;
            for (int k = 0; k < nb; ++k)
                tau[k] += s.nH * (xs[0] * b.sH[k] + s.yHe * (xs[1] * b.sHe1[k] + xs[2] * b.sHe2[k])) * dr_cm;
        }
        double dmax = 0.0;
        for (int i = 0; i < nr; ++i) dmax = std::max(dmax, std::fabs(Te[i] / prev[i] - 1.0));
        if (dmax < 1.0e-6) break;
    }
    return 0;
}

}  // namespace orc
