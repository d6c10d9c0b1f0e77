// Host set-up of the thermal-balance tables: the thermally averaged
// free-free Gaunt factor (cooling_mod.f90:80-86, 182-220, with the Hummer
// (1988) expansion of gaunt.f90), the H I collisional line-cooling fit
// (cooling_mod.f90:73-75, 98-134) and its (T, n_e) n-level suppression
// table (nlevel_cooling_mod.f90 over the nlevel_mod.f90 solver).
#include "thermal.h"
#include "species.h"

#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "physics.cuh"

namespace mochii {

namespace {

// Hummer (1988, ApJ 327, 477) two-dimensional Chebyshev coefficients of the
// thermally averaged free-free Gaunt factor, column-major (8 x 11).
const double kHummer[88] = {
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

// Gaunt factor g_ff(u) at one temperature for an array of log10(h nu/Ryd),
// in the single-precision arithmetic the reference evaluates it with: the
// temperature-dependent Chebyshev coefficients c_j (Clenshaw in txg) and the
// u expansion, with the limiting forms outside the fitted wedge.
void hummer_gff(float log10z, float log10T, const float* xlf, int n, float* g) {
    const float xlrkt = log10T < 2.5f ? 5.1983649f - 2.5f : log10T > 8.f ? 5.1983649f - 8.f : 5.1983649f - log10T;
    const float txg = 0.66666667f * (2.0f * log10z + xlrkt);
    const float gamma2 = powf(10.0f, txg * 1.5f);
    const float con = 0.72727273f * xlrkt + 0.90909091f;
    float c[9];
    for (int j = 1; j <= 8; ++j) {
        float b[12];
        b[11] = (float)kHummer[80 + j - 1];
        b[10] = (float)((double)(txg * b[11]) + kHummer[72 + j - 1]);
        for (int r = 9; r >= 1; --r) b[r] = (float)((double)(txg * b[r + 1] - b[r + 2]) + kHummer[(r - 1) * 8 + j - 1]);
        c[j] = 0.25f * (b[1] - b[3]);
    }
    for (int i = 0; i < n; ++i) {
        const float txu = 0.72727273f * xlf[i] + con;
        const float u = powf(10.0f, (txu - .90909091f) / .72727273f);
        float r = 0.0f;
        if (std::fabs(txu) <= 2.0f) {
            float b[9];
            b[8] = c[8];
            b[7] = txu * b[8] + c[7];
            for (int k = 6; k >= 1; --k) b[k] = txu * b[k + 1] - b[k + 2] + c[k];
            r = b[1] - b[3];
        } else if (log10f(u) < -4.0f) {
            r = gamma2 < 0.3f ? 0.551329f * logf(2.24593f / u) : 0.551329f * logf(0.944931f / u / sqrtf(gamma2));
        } else if (txu > 2.0f) {
            if (log10f(gamma2) < -3.f) {
                r = sqrtf(0.9549297f / u);
            } else if (log10f(gamma2) < 0.0f) {
                const float slope = (sqrtf(12 * gamma2 / u) - sqrtf(0.9549297f / u)) / 3.0f;
                r = sqrtf(12 * gamma2 / u) + slope * log10f(gamma2);
            } else {
                r = std::fmin(1.05f, sqrtf(12.f * gamma2 / u));
            }
        }
        g[i] = r;
    }
}

// Thermal average <g_ff> = int g(u) e^-u du over a 64-point log-u midpoint
// grid on [1e-4, 20], normalised by the same range's int e^-u du.
double gff_mean(double T, double Z) {
    const int NU = 64;
    const double lo = std::log(1.0e-4), hi = std::log(20.0);
    const double ryd_kt = 13.605693 * kEv2erg / (kKboltz * T);
    double u[NU], du[NU];
    float xlf[NU], g[NU];
    for (int i = 0; i < NU; ++i) {
        u[i] = std::exp(lo + (hi - lo) * ((double)(i + 1) - 0.5) / (double)NU);
        du[i] = u[i] * (hi - lo) / (double)NU;
        xlf[i] = (float)std::log10(u[i] / ryd_kt);
    }
    hummer_gff((float)std::log10(Z), (float)std::log10(T), xlf, NU, g);
    double s = 0.0;
    for (int i = 0; i < NU; ++i) s = s + (double)g[i] * std::exp(-u[i]) * du[i];
    return s / (std::exp(-1.0e-4) - std::exp(-20.0));
}

}  // namespace

bool cooling_fit_read(const std::string& path, std::vector<double>& A, std::vector<double>& Ti) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    int n = -1;
    while (std::getline(f, line)) {
        const size_t a = line.find_first_not_of(" \t");
        if (a == std::string::npos || line[a] == '#') continue;
        n = std::atoi(line.c_str() + a);
        break;
    }
    if (n < 1 || n > kMaxFitTerms) return false;
    A.resize(n);
    Ti.resize(n);
    for (int i = 0; i < n; ++i)
        if (!(f >> A[i] >> Ti[i])) return false;
    return true;
}

std::string data_root() {
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&data_root), &info) && info.dli_fname) {
        std::string p(info.dli_fname);
        const size_t s = p.find_last_of('/');
        if (s != std::string::npos) return p.substr(0, s) + "/data";
    }
    return "data";
}

std::string atomic_dir(const mochii_params& p) {
    if (p.atomic_dir[0]) return p.atomic_dir;
    if (p.data_dir[0]) return std::string(p.data_dir) + "/atomic";
    return data_root() + "/atomic";
}

// n-level atom file (nlevel_mod.f90:61-105 layout: NLEV / NRAD / NUPS blocks).
bool NlevelAtomData::load(const std::string& path) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
        const size_t a = line.find_first_not_of(" \t");
        if (a == std::string::npos || line[a] == '#') continue;
        std::istringstream ss(line);
        std::string key;
        int n = 0;
        ss >> key >> n;
        if (key == "NLEV") {
            if (n > kMaxLev) return false;
            g.resize(n);
            e_cm1.resize(n);
            for (int k = 0; k < n; ++k) {
                int idx;
                f >> idx >> g[k] >> e_cm1[k];
            }
            std::getline(f, line);
        } else if (key == "NRAD") {
            rad.resize(n);
            for (auto& r : rad) f >> r.l >> r.u >> r.A;
            std::getline(f, line);
        } else if (key == "NUPS") {
            ups.resize(n);
            for (auto& u : ups) {
                std::getline(f, line);
                std::istringstream ls(line);
                int nc;
                ls >> u.l >> u.u >> u.type >> u.C >> u.dE >> u.st_lo >> u.st_hi >> u.logf >> nc;
                u.c.resize(nc);
                for (auto& x : u.c) ls >> x;
            }
        }
    }
    return !g.empty() && !ups.empty();
}

// Effective collision strength from the Burgess-Tully scaled Chebyshev fit
// (the recipe of the n-level files, nlevel_mod.f90:119-152).
double NlevelAtomData::upsilon(const Ups& u, double T) {
    const double et = (kKboltz / 2.1798723611035e-11) * T / u.dE;
    double st = (u.type == 1 || u.type == 4) ? 1.0 - std::log(u.C) / std::log(et + u.C) : et / (et + u.C);
    st = std::min(std::max(st, u.st_lo), u.st_hi);
    const double x = u.st_hi > u.st_lo ? 2.0 * (st - u.st_lo) / (u.st_hi - u.st_lo) - 1.0 : 0.0;
    double b0 = 0.0, b1 = 0.0;
    for (int j = (int)u.c.size() - 1; j >= 1; --j) {
        const double b2 = b1;
        b1 = b0;
        b0 = 2.0 * x * b1 - b2 + u.c[j];
    }
    double y = x * b0 - b1 + u.c[0];
    if (u.logf == 1) y = std::pow(10.0, y);
    double r;
    switch (u.type) {
        case 1: r = y * std::log(et + std::exp(1.0)); break;
        case 2: r = y; break;
        case 3: r = y / (et + 1.0); break;
        case 4: r = y * std::log(et + u.C); break;
        case 5: r = y / et; break;
        default: r = std::pow(10.0, y); break;
    }
    return std::max(r, 0.0);
}

// Collisional line-cooling coefficient Lambda_SE(T, n_e) = sum n_u A dE / n_e
// from statistical equilibrium (collisions + spontaneous decay, closure
// sum n = 1, Gaussian elimination with partial pivoting); every pair is
// oriented by level energy (nlevel_mod.f90:168-181, 247-326).
void NlevelAtomData::cooling_column(double T, const double* ne, int nne, double* out) const {
    const int n = (int)g.size();
    const double hc = 1.9864458571489287e-16;
    std::vector<double> Rc((size_t)n * n, 0.0), Rr((size_t)n * n, 0.0);
    auto orient = [&](int i1, int i2, int& lo, int& hi) {
        if (e_cm1[i2 - 1] >= e_cm1[i1 - 1]) { lo = i1; hi = i2; } else { lo = i2; hi = i1; }
    };
    for (const Ups& u : ups) {
        int lo, hi;
        orient(u.l, u.u, lo, hi);
        const double de = (e_cm1[hi - 1] - e_cm1[lo - 1]) * hc;
        const double q_ul = 8.629e-6 / (g[hi - 1] * std::sqrt(T)) * upsilon(u, T);
        const double q_lu = (g[hi - 1] / g[lo - 1]) * q_ul * std::exp(-de / (kKboltz * T));
        Rc[(size_t)(hi - 1) * n + (lo - 1)] += q_lu;
        Rc[(size_t)(lo - 1) * n + (hi - 1)] += q_ul;
    }
    for (const Rad& r : rad) {
        int lo, hi;
        orient(r.l, r.u, lo, hi);
        Rr[(size_t)(lo - 1) * n + (hi - 1)] += r.A;
    }
    std::vector<double> M((size_t)n * (n + 1)), pop(n);
    for (int jn = 0; jn < nne; ++jn) {
        const double e = ne[jn];
        auto R = [&](int i, int j) { return e * Rc[(size_t)i * n + j] + Rr[(size_t)i * n + j]; };
        std::fill(M.begin(), M.end(), 0.0);
        auto m = [&](int i, int j) -> double& { return M[(size_t)i * (n + 1) + j]; };
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                if (i != j) {
                    m(i, j) = R(i, j);
                    m(i, i) = m(i, i) - R(j, i);
                }
        for (int j = 0; j < n; ++j) m(0, j) = 1.0;
        m(0, n) = 1.0;
        for (int i = 0; i < n - 1; ++i) {
            int ip = i;
            for (int j = i + 1; j < n; ++j)
                if (std::fabs(m(j, i)) > std::fabs(m(ip, i))) ip = j;
            if (ip != i)
                for (int j = i; j <= n; ++j) std::swap(m(i, j), m(ip, j));
            for (int j = i + 1; j < n; ++j) {
                const double fac = m(j, i) / m(i, i);
                for (int k = i; k <= n; ++k) m(j, k) = m(j, k) - fac * m(i, k);
            }
        }
        for (int i = n - 1; i >= 0; --i) {
            double p = m(i, n);
            for (int j = i + 1; j < n; ++j) p = p - m(i, j) * pop[j];
            pop[i] = p / m(i, i);
        }
        double lam = 0.0;
        for (const Rad& r : rad) {
            int lo, hi;
            orient(r.l, r.u, lo, hi);
            lam = lam + pop[hi - 1] * r.A * ((e_cm1[hi - 1] - e_cm1[lo - 1]) * hc);
        }
        out[jn] = lam / e;
    }
}

bool thermal_tables_build(const mochii_params& p, ThermalHost& t, std::string* err) {
    for (int i = 0; i < kGffNT; ++i) {
        t.gff_logT[i] = 2.0 + 4.0 * (double)i / (double)(kGffNT - 1);
        for (int z = 0; z < kGffNZ; ++z) t.gff[i * kGffNZ + z] = gff_mean(std::pow(10.0, t.gff_logT[i]), (double)(z + 1));
    }
    const std::string dir = atomic_dir(p);
    std::vector<double> A, Ti;
    if (!cooling_fit_read(dir + "/cooling_h_1.txt", A, Ti)) {
        if (err) *err = "cannot read " + dir + "/cooling_h_1.txt";
        return false;
    }
    t.hi_nterm = (int)A.size();
    for (int i = 0; i < t.hi_nterm; ++i) { t.hi_A[i] = A[i]; t.hi_T[i] = Ti[i]; }
    t.use_hi_table = p.cooling_local_ne;
    // nlevel_cooling_add returns 0 without the atom file: the fit is used unchanged
    if (t.use_hi_table) t.use_hi_table = nlevel_table_build(dir + "/nlevel_h_1.txt", t.hi_lamref, t.hi_Ssup);
    return true;
}

bool nlevel_table_build(const std::string& path, std::vector<double>& lamref, std::vector<double>& Ssup) {
    NlevelAtomData atom;
    if (!atom.load(path)) return false;
    std::vector<double> ne(kNlNNE), lam((size_t)kNlNT * kNlNNE);
    for (int j = 0; j < kNlNNE; ++j) ne[j] = std::pow(10.0, -6.0 + 0.1 * (double)j);
    for (int i = 0; i < kNlNT; ++i)
        atom.cooling_column(std::pow(10.0, 2.0 + 0.01 * (double)i), ne.data(), kNlNNE, &lam[(size_t)i * kNlNNE]);
    lamref.resize(kNlNT);
    Ssup.resize((size_t)kNlNT * kNlNNE);
    for (int i = 0; i < kNlNT; ++i) {
        const double ref = lam[(size_t)i * kNlNNE];
        lamref[i] = ref;
        for (int j = 0; j < kNlNNE; ++j) Ssup[(size_t)i * kNlNNE + j] = lam[(size_t)i * kNlNNE + j] / std::max(ref, kTinest);
    }
    return true;
}

}  // namespace mochii
