// Tabulated source spectra and the analytic ISRF presets: the spectrum
// files of every source slot (read_shape_table / read_phys_table,
// ion_band_mod.f90:1438-1597), the band-clipped tabulated sampler
// (build_tabulated_band_sampler, energy_sampler_mod.f90:66-104, 336-359) and
// the Draine, Habing and Mathis fields (ion_band_mod.f90:895-911,
// 1627-1720).  Set-up time only, on the host.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "band.h"
#include "physics.cuh"

namespace mochii {

namespace {

constexpr double kHcEvAng = 12398.42;   // eV Angstrom (define.f90:62)
constexpr int kPresetN = 4096;          // NPRESET (ion_band_mod.f90:105)
constexpr double kPresetEmax = 13.6;    // PRESET_EMAX: the presets carry no flux above it

bool fail(std::string* err, const std::string& m) {
    if (err) *err = m;
    return false;
}

// Fortran list-directed values of one line: blanks and commas separate,
// a D exponent reads as E.
std::vector<double> line_values(std::string s) {
    for (auto& ch : s) {
        if (ch == ',' || ch == '\t') ch = ' ';
        else if (ch == 'd' || ch == 'D') ch = 'e';
    }
    std::vector<double> v;
    const char* p = s.c_str();
    for (;;) {
        while (*p == ' ') ++p;
        if (!*p) break;
        char* end = nullptr;
        const double x = std::strtod(p, &end);
        if (end == p) break;
        v.push_back(x);
        p = end;
    }
    return v;
}

// linear_table_value (energy_sampler_mod.f90:336-359).
double linear_value(const std::vector<double>& e, const std::vector<double>& f, double v) {
    const int n = (int)e.size();
    if (v <= e[0]) return f[0];
    if (v >= e[n - 1]) return f[n - 1];
    int lo = 1, hi = n;   // 1-based bracket, bisection as the reference's
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (e[mid - 1] <= v) lo = mid; else hi = mid;
    }
    const double fr = (v - e[lo - 1]) / (e[hi - 1] - e[lo - 1]);
    return f[lo - 1] + fr * (f[hi - 1] - f[lo - 1]);
}

// Draine (1978) FUV field J_E [erg/s/cm^2/sr/eV] on 5-13.6 eV: the photon
// fit E N(E) = 1.658e6 E^2 - 2.152e5 E^3 + 6.919e3 E^4 times eV in erg.
double draine_je(double E) {
    if (E < 5.0 || E > 13.6) return 0.0;
    const double e2 = E * E;   // integer powers as repeated squaring: E^3 = E^2 E, E^4 = (E^2)^2
    const double fph = 1.658e6 * e2 - 2.152e5 * (e2 * E) + 6.919e3 * (e2 * e2);
    return kEv2erg * fph;
}

// Planck B_lambda [W m^-2 m^-1 sr^-1] at lambda [um] in SI constants.
double bbody_si(double T, double lam_um) {
    const double c = 2.99792458e8, h = 6.62606957e-34, kb = 1.3806488e-23;
    const double hc2 = (2.0 * h) * (c * c), hckb = h * c / kb;
    if (T <= 0.0 || lam_um <= 0.0) return 0.0;
    const double lam = lam_um * 1.0e-6;
    const double x = hckb / (T * lam);
    if (x >= 700.0) return 0.0;
    const double l2 = lam * lam, l5 = (l2 * l2) * lam;
    return hc2 / l5 / (std::exp(x) - 1.0);
}

// Mathis, Mezger & Panagia (1983) J_lambda [W m^-2 m^-1 sr^-1] at lambda
// [um]: UV power laws and three diluted blackbodies.
double mathis_jl_si(double lam_um) {
    if (lam_um < 0.0912) return 0.0;
    if (lam_um < 0.110) return 3069.0 * std::pow(lam_um, 3.4172);
    if (lam_um < 0.134) return 1.627;
    if (lam_um < 0.250) return 0.0566 * std::pow(lam_um, -1.6678);
    return 1.0e-14 * bbody_si(7500.0, lam_um) + 1.65e-13 * bbody_si(4000.0, lam_um) +
           4.0e-13 * bbody_si(3000.0, lam_um);
}

// J_E = J_lambda(SI) x 10 (W m^-2 m^-1 -> erg s^-1 cm^-2 cm^-1) x hc / E^2.
double mathis_je(double E) {
    const double lam_um = kHcEvAng * 1.0e-4 / E;
    return mathis_jl_si(lam_um) * (kHcEvAng * 1.0e-7) / (E * E);
}

}  // namespace

int spectrum_preset_id(const char* name) {
    std::string s(name ? name : "");
    const size_t a = s.find_first_not_of(' ');
    s = a == std::string::npos ? std::string() : s.substr(a);
    while (!s.empty() && s.back() == ' ') s.pop_back();
    for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch);
    if (s == "draine") return 1;
    if (s == "habing") return 2;
    if (s == "mathis") return 3;
    return 0;
}

double preset_je(double E, int id) {
    if (id == 1) return draine_je(E);
    if (id == 2) return draine_je(E) / 1.71;
    if (id == 3) return mathis_je(E);
    return 0.0;
}

bool spectrum_read(const std::string& path, int icol, int ncol, int type, std::vector<double>& e,
                   std::vector<double>& f, std::string* err) {
    FILE* fp = std::fopen(path.c_str(), "r");
    if (!fp) return fail(err, "cannot open " + path);
    e.clear();
    f.clear();
    char buf[4096];
    while (std::fgets(buf, sizeof(buf), fp)) {
        std::string line(buf);
        const size_t a = line.find_first_not_of(" \t\r\n");
        if (a == std::string::npos || line[a] == '#') continue;
        const std::vector<double> v = line_values(line.substr(a));
        if ((int)v.size() < ncol + 1) {
            std::fclose(fp);
            return fail(err, path + " needs 1 + " + std::to_string(ncol) + " columns (the first the abscissa)");
        }
        const double c1 = v[0], cv = v[icol];
        double ee = c1, xe = cv;
        if (type == 2) {          // per_hz: E = h nu / e, X_E = X_nu e / h
            ee = kHPlanck * c1 / kEv2erg;
            xe = cv * kEv2erg / kHPlanck;
        } else if (type == 3) {   // per_ang: E = hc / lambda, X_E = X_lambda hc / E^2
            ee = kHcEvAng / c1;
            xe = cv * kHcEvAng / (ee * ee);
        } else if (type == 4) {   // per_um
            const double hc = kHcEvAng * 1.0e-4;
            ee = hc / c1;
            xe = cv * hc / (ee * ee);
        }
        e.push_back(ee);
        f.push_back(xe);
    }
    std::fclose(fp);
    // ascending in E (wavelength tables arrive descending): insertion sort
    for (size_t i = 1; i < e.size(); ++i)
        for (size_t j = i; j >= 1; --j) {
            if (e[j - 1] <= e[j]) break;
            std::swap(e[j - 1], e[j]);
            std::swap(f[j - 1], f[j]);
        }
    return true;
}

bool table_band(EnergyTable& t, const std::vector<double>& e, const std::vector<double>& f, double emin, double emax,
                std::string* err) {
    const size_t n = e.size();
    if (n < 2 || f.size() != n) return fail(err, "energy sampler: table needs at least two matching columns");
    for (size_t i = 0; i < n; ++i)
        if (f[i] < 0.0) return fail(err, "energy sampler: negative spectral density");
    for (size_t i = 1; i < n; ++i)
        if (e[i] <= e[i - 1]) return fail(err, "energy sampler: energies must be strictly ascending");
    if (emax <= emin) return fail(err, "energy sampler: invalid requested band");
    const double lo = std::max(emin, e[0]), hi = std::min(emax, e[n - 1]);
    if (hi <= lo) return fail(err, "energy sampler: table does not overlap requested band");
    std::vector<double> ce{lo}, cf{linear_value(e, f, lo)};
    for (size_t i = 0; i < n; ++i)
        if (e[i] > lo && e[i] < hi) {
            ce.push_back(e[i]);
            cf.push_back(f[i]);
        }
    ce.push_back(hi);
    cf.push_back(linear_value(e, f, hi));
    return table_from_points(t, ce, cf, err);
}

bool preset_table(EnergyTable& t, int id, double elo, double emax, double scale, std::string* err) {
    const double ehi = std::min(emax, kPresetEmax);
    if (ehi <= elo) return fail(err, "the ISRF preset carries no flux above 13.6 eV, so it does not overlap the band");
    std::vector<double> e(kPresetN), f(kPresetN);
    for (int k = 0; k < kPresetN; ++k) {
        e[k] = elo + (ehi - elo) * (double)k / (double)(kPresetN - 1);
        f[k] = preset_je(e[k], id) * scale;
    }
    return table_from_points(t, e, f, err);
}

}  // namespace mochii
