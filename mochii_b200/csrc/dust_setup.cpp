// Host read of the grain extinction table (gas_opacity_mod.f90 ion_dust_read,
// :69-121).  Fortran reads each line list-directed into four reals and keeps
// the line when that succeeds and lambda > 0; a token counts as a real in
// the forms F editing accepts (1.5, 1.5E3, 1.5D3, and 1.5-3 = 1.5E-3).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <numeric>
#include <sstream>

#include "dust.h"

namespace mochii {

namespace {

bool real_token(const std::string& tok, double* v) {
    if (tok.empty()) return false;
    std::string t;
    t.reserve(tok.size() + 1);
    for (size_t k = 0; k < tok.size(); ++k) {
        char ch = tok[k];
        if (ch == 'd' || ch == 'D') ch = 'E';
        // a signed exponent without its letter
        if (k > 0 && (ch == '+' || ch == '-') && t.back() != 'E' && t.back() != 'e') t.push_back('E');
        t.push_back(ch);
    }
    char* end = nullptr;
    const double x = std::strtod(t.c_str(), &end);
    if (end == t.c_str() || *end != '\0') return false;
    *v = x;
    return true;
}

double log_interp(const DustHost& d, const std::vector<double>& y, double x0) {
    const std::vector<double>& x = d.lam;
    const size_t n = x.size();
    if (x0 <= x[0]) return y[0];
    if (x0 >= x[n - 1]) return y[n - 1];
    const size_t i = (size_t)(std::upper_bound(x.begin(), x.end(), x0) - x.begin()) - 1;
    const double w = std::log(x0 / x[i]) / std::log(x[i + 1] / x[i]);
    return std::exp(std::log(std::max(y[i], 1.0e-300)) * (1.0 - w) + std::log(std::max(y[i + 1], 1.0e-300)) * w);
}

}  // namespace

bool dust_table_read(const std::string& path, double lambda_ref, DustHost& d, std::string* err) {
    std::ifstream f(path);
    if (!f) {
        if (err) *err = "ion_add_dust needs par%ion_dust_kext; cannot open " + path;
        return false;
    }
    std::vector<double> lam, alb, gcos, cext;
    std::string line;
    while (std::getline(f, line)) {
        const size_t slash = line.find('/');   // a slash ends a list-directed record
        if (slash != std::string::npos) line.resize(slash);
        std::replace(line.begin(), line.end(), ',', ' ');
        std::replace(line.begin(), line.end(), '\t', ' ');
        std::istringstream s(line);
        std::string tok;
        double v[4];
        int nv = 0;
        while (nv < 4 && (s >> tok) && real_token(tok, &v[nv])) ++nv;
        if (nv < 4 || !(v[0] > 0.0)) continue;
        lam.push_back(v[0]);
        alb.push_back(v[1]);
        gcos.push_back(v[2]);
        cext.push_back(v[3]);
    }
    if (lam.size() < 2) {
        if (err) *err = path + ": fewer than two extinction rows";
        return false;
    }
    std::vector<size_t> ord(lam.size());
    std::iota(ord.begin(), ord.end(), (size_t)0);
    std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return lam[a] < lam[b]; });
    d = DustHost();
    for (size_t k : ord) {
        d.lam.push_back(lam[k]);
        d.alb.push_back(alb[k]);
        d.gcos.push_back(gcos[k]);
        d.cext.push_back(cext[k]);
    }
    d.cref = log_interp(d, d.cext, lambda_ref);
    if (!(d.cref > 0.0)) {
        if (err) *err = path + ": C_ext at par%lambda_ref is not positive";
        return false;
    }
    return true;
}

}  // namespace mochii
