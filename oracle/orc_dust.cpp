// Oracle (test infrastructure only): gas_opacity_mod.f90 grain optics and
// the Philox4x32-10 packet streams.
#include "orc_dust.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <numeric>
#include <sstream>

namespace orc {

static constexpr double TINEST_D = 1.0e-300;   // define.f90 tinest

bool fortran_real(const std::string& tok, double* v) {
    if (tok.empty()) return false;
    std::string t = tok;
    for (char& c : t)
        if (c == 'd' || c == 'D') c = 'E';
    // an exponent written as a bare sign (F editing: "1.5-3" = 1.5E-3)
    size_t k = 1;
    for (; k < t.size(); ++k)
        if ((t[k] == '+' || t[k] == '-') && t[k - 1] != 'E' && t[k - 1] != 'e') break;
    if (k < t.size()) t.insert(k, "E");
    const char* s = t.c_str();
    char* end = nullptr;
    const double x = std::strtod(s, &end);
    if (end == s || *end != '\0') return false;
    *v = x;
    return true;
}

bool DustTable::read(const std::string& path, double lambda_ref, std::string* err) {
    std::ifstream f(path);
    if (!f) {
        if (err) *err = "ion_add_dust needs par%ion_dust_kext; cannot open " + path;
        return false;
    }
    lam.clear(); alb.clear(); gcos.clear(); cext.clear();
    std::string line;
    while (std::getline(f, line)) {
        // list-directed read of four reals: separators are blanks and commas;
        // a slash ends the record
        for (char& c : line)
            if (c == ',' || c == '\t') c = ' ';
        const size_t sl = line.find('/');
        if (sl != std::string::npos) line = line.substr(0, sl);
        std::istringstream s(line);
        std::string tok;
        double v[4];
        int nv = 0;
        while (nv < 4 && (s >> tok)) {
            if (!fortran_real(tok, &v[nv])) break;
            ++nv;
        }
        if (nv < 4 || !(v[0] > 0.0)) continue;
        lam.push_back(v[0]); alb.push_back(v[1]); gcos.push_back(v[2]); cext.push_back(v[3]);
    }
    if (lam.size() < 2) {
        if (err) *err = path + ": fewer than two extinction rows";
        return false;
    }
    // sort4: stable ascending in lambda
    std::vector<size_t> ord(lam.size());
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return lam[a] < lam[b]; });
    auto perm = [&](std::vector<double>& a) {
        std::vector<double> o(a.size());
        for (size_t i = 0; i < a.size(); ++i) o[i] = a[ord[i]];
        a.swap(o);
    };
    perm(lam); perm(alb); perm(gcos); perm(cext);
    cref = interp_log(lam, cext, lambda_ref);
    return true;
}

double interp_log(const std::vector<double>& x, const std::vector<double>& y, double x0) {
    const size_t n = x.size();
    if (x0 <= x[0]) return y[0];
    if (x0 >= x[n - 1]) return y[n - 1];
    size_t i = 0;
    for (; i < n - 1; ++i)
        if (x0 < x[i + 1]) break;
    const double w = std::log(x0 / x[i]) / std::log(x[i + 1] / x[i]);
    return std::exp(std::log(std::max(y[i], TINEST_D)) * (1.0 - w) + std::log(std::max(y[i + 1], TINEST_D)) * w);
}

double interp_lin(const std::vector<double>& x, const std::vector<double>& y, double x0) {
    const size_t n = x.size();
    if (x0 <= x[0]) return y[0];
    if (x0 >= x[n - 1]) return y[n - 1];
    size_t i = 0;
    for (; i < n - 1; ++i)
        if (x0 < x[i + 1]) break;
    const double w = (x0 - x[i]) / (x[i + 1] - x[i]);
    return y[i] * (1.0 - w) + y[i + 1] * w;
}

// ---- dust_temp_mod.f90 --------------------------------------------------
double planck_nu(double nu, double T) {   // :118-127
    const double x = 6.62607015e-27 * nu / (1.380649e-16 * T);
    return x < 700.0 ? 2.0 * 6.62607015e-27 * nu * nu * nu / (2.99792458e10 * 2.99792458e10) / (std::exp(x) - 1.0)
                     : 0.0;
}

void DustTemp::setup(const DustTable& d) {   // dust_temp_setup, :38-115
    const double c = 2.99792458e10, fourpi = 12.566370614359172953850573533118;
    for (int k = 0; k < NIR; ++k) {
        lam_ir[k] = std::exp(std::log(1.0) + (std::log(1000.0) - std::log(1.0)) * (double)k / (double)(NIR - 1));
        sabs_ir[k] = (1.0 - interp_lin(d.lam, d.alb, lam_ir[k])) * interp_log(d.lam, d.cext, lam_ir[k]) / d.cref;
    }
    const size_t n = d.lam.size();
    for (int i = 0; i < NT; ++i) {
        tgrid[i] = std::pow(10.0, 0.5 + 3.0 * (double)i / (double)(NT - 1));
        const double T = tgrid[i];
        double f = 0.0;
        for (size_t k = 0; k + 1 < n; ++k) {
            const double nu1 = c / (d.lam[k + 1] * 1.0e-4), nu2 = c / (d.lam[k] * 1.0e-4);
            const double snu = 0.5 * ((1.0 - d.alb[k]) * d.cext[k] + (1.0 - d.alb[k + 1]) * d.cext[k + 1]) / d.cref;
            const double bnu = 0.5 * (planck_nu(nu1, T) + planck_nu(nu2, T));
            f = f + fourpi * snu * bnu * (nu2 - nu1);
        }
        femit[i] = f;
    }
}

double DustTemp::femit_of(double T) const {   // :129-135
    const double lt = std::min(std::max(std::log10(T), std::log10(tgrid[0])), std::log10(tgrid[NT - 1]));
    const int i = std::min((int)((lt - std::log10(tgrid[0])) / (3.0 / (double)(NT - 1))) + 1, NT - 1) - 1;
    const double w = (lt - std::log10(tgrid[i])) / (std::log10(tgrid[i + 1]) - std::log10(tgrid[i]));
    return std::exp(std::log(femit[i]) * (1.0 - w) + std::log(femit[i + 1]) * w);
}

double DustTemp::solve(double kd, double heat) const {   // dust_temp_compute, :137-170
    if (kd <= 0.0 || heat <= 0.0) return 0.0;
    const double target = heat / kd;
    double tlo = tgrid[0], thi = tgrid[NT - 1];
    if (femit_of(thi) <= target) return thi;
    for (int it = 0; it < 60; ++it) {
        const double tm = std::sqrt(tlo * thi);
        if (femit_of(tm) < target) tlo = tm;
        else thi = tm;
        if (thi / tlo - 1.0 < 1.0e-5) break;
    }
    return std::sqrt(tlo * thi);
}

double DustTable::sabs_at(double E) const {
    const double lb = 1.23984 / E;
    return (1.0 - interp_lin(lam, alb, lb)) * interp_log(lam, cext, lb) / cref;
}
double DustTable::ssca_at(double E) const {
    const double lb = 1.23984 / E;
    return interp_lin(lam, alb, lb) * interp_log(lam, cext, lb) / cref;
}
double DustTable::g_at(double E) const { return interp_lin(lam, gcos, 1.23984 / E); }

// ---- Philox4x32-10 -----------------------------------------------------------
static inline void mulhilo(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
}

void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo(0xD2511F53u, c0, &hi0, &lo0);
        mulhilo(0xCD9E8D57u, c2, &hi1, &lo1);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

double philox_uniform(uint64_t seed, uint32_t stream, uint64_t packet, uint32_t n) {
    const uint32_t ctr[4] = {n >> 1, 0u, (uint32_t)packet, (uint32_t)(packet >> 32)};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ stream};
    uint32_t o[4];
    philox4x32_10(ctr, key, o);
    const uint32_t a = (n & 1) ? o[2] : o[0], b = (n & 1) ? o[3] : o[1];
    const uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);   // 53 bits
    return ((double)m + 0.5) * (1.0 / 9007199254740992.0);
}

}  // namespace orc
