// Host set-up of the trace-metal registry: element files
// (read_element, species_mod.f90:358-423), the registry order and the
// threshold sort of species_setup (species_mod.f90:143-226), per-stage
// cooling fits and their n-level (T, n_e) suppression tables
// (nlevel_cooling_add, nlevel_cooling_mod.f90:104-163).
#include "species.h"

#include "metals.cuh"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>
#include <thread>

namespace mochii {

namespace {

struct ElementFile {
    std::string name;
    int Z = 0, nstage = 0;
    double eth[kMaxSt] = {};
    int photo_form[kMaxSt] = {1, 1, 1, 1, 1, 1};
    double photo[kMaxSt][8] = {};
    double ci[kMaxSt][5] = {}, rr[kMaxSt][6] = {};
    int ndr[kMaxSt] = {};
    double dr_c[kMaxSt][9] = {}, dr_e[kMaxSt][9] = {};
    int has_dr2[kMaxSt] = {}, has_rr2[kMaxSt] = {};
    double dr2[kMaxSt][4] = {}, rr2[kMaxSt][2] = {};
    int cxi_form[kMaxSt] = {}, cxr_form[kMaxSt] = {};
    double cxi[kMaxSt][6] = {}, cxr[kMaxSt][6] = {};
};

bool parse_element(const std::string& path, ElementFile& e, std::string* err) {
    std::ifstream f(path);
    if (!f) {
        if (err) *err = "cannot open " + path;
        return false;
    }
    std::string line;
    int it = 0;
    auto bad = [&](const std::string& what) {
        if (err) *err = path + ": " + what;
        return false;
    };
    while (std::getline(f, line)) {
        const size_t a = line.find_first_not_of(" \t\r");
        if (a == std::string::npos || line[a] == '#') continue;
        std::istringstream s(line.substr(a));
        std::string key;
        s >> key;
        if (key == "ELEMENT") {
            if (!(s >> e.name >> e.Z >> e.nstage) || e.nstage < 1 || e.nstage > kMaxSt) return bad("bad ELEMENT line");
            continue;
        }
        if (key == "TRANSITION") {
            if (!(s >> it) || it < 1 || it >= kMaxSt) return bad("bad TRANSITION line");
            continue;
        }
        if (it < 1) continue;
        const int k = it - 1;
        bool ok = true;
        if (key == "ETH") {
            ok = (bool)(s >> e.eth[k]);
        } else if (key == "PHOTO" || key == "PHOTO2") {
            const int n = key == "PHOTO" ? 8 : 7;
            for (int j = 0; j < n; ++j) ok = ok && (bool)(s >> e.photo[k][j]);
            e.photo_form[k] = key == "PHOTO" ? 1 : 2;
        } else if (key == "CI") {
            for (int j = 0; j < 5; ++j) ok = ok && (bool)(s >> e.ci[k][j]);
        } else if (key == "RR") {
            for (int j = 0; j < 6; ++j) ok = ok && (bool)(s >> e.rr[k][j]);
        } else if (key == "DR") {
            int n = 0;
            ok = (bool)(s >> n) && n >= 0 && n <= 9;
            e.ndr[k] = ok ? n : 0;
            for (int j = 0; ok && j < n; ++j) ok = (bool)(s >> e.dr_c[k][j]);
            for (int j = 0; ok && j < n; ++j) ok = (bool)(s >> e.dr_e[k][j]);
        } else if (key == "DR2") {
            for (int j = 0; j < 4; ++j) ok = ok && (bool)(s >> e.dr2[k][j]);
            e.has_dr2[k] = 1;
        } else if (key == "RR2") {
            for (int j = 0; j < 2; ++j) ok = ok && (bool)(s >> e.rr2[k][j]);
            e.has_rr2[k] = 1;
        } else if (key == "CXI" || key == "CXR") {
            int& form = key == "CXI" ? e.cxi_form[k] : e.cxr_form[k];
            double* c = key == "CXI" ? e.cxi[k] : e.cxr[k];
            ok = (bool)(s >> form);
            if (ok && form > 0)
                for (int j = 0; j < 6; ++j) ok = ok && (bool)(s >> c[j]);
        }
        if (!ok) return bad("bad " + key + " line");
    }
    if (e.nstage < 1) return bad("no ELEMENT line");
    return true;
}

// ci_dere_ratio (recomb_mod.f90): Dere (2007) / Voronov (1997) rate ratio at
// 1e4 K per (Z, stage) under par%ci_model = 'dere_hybrid', 1 otherwise.
double dere_ratio(int Z, int stage, bool hybrid) {
    if (!hybrid) return 1.0;
    double t[4] = {1, 1, 1, 1};
    int n = 0;
    switch (Z) {
        case 6: t[0] = 1.0499; t[1] = 0.913; t[2] = 1.0377; n = 3; break;
        case 7: t[0] = 1.0421; t[1] = 1.1966; n = 2; break;
        case 8: t[0] = 1.041; t[1] = 1.1181; n = 2; break;
        case 10: t[0] = 0.8089; t[1] = 1.1395; n = 2; break;
        case 12: t[0] = 0.3793; t[1] = 0.9857; n = 2; break;
        case 14: t[0] = 0.7328; t[1] = 0.8798; t[2] = 0.4492; t[3] = 0.8221; n = 4; break;
        case 16: t[0] = 1.3572; t[1] = 0.8925; t[2] = 0.8119; n = 3; break;
        case 17: t[0] = 0.5412; t[1] = 0.8428; t[2] = 0.9237; t[3] = 0.819; n = 4; break;
        case 18: t[0] = 0.9242; t[1] = 0.8644; t[2] = 0.9752; n = 3; break;
        case 20: t[0] = 0.7652; t[1] = 1.1668; t[2] = 1.0422; t[3] = 0.8705; n = 4; break;
        case 26: t[0] = 0.9904; t[1] = 1.0568; t[2] = 1.824; n = 3; break;
        default: break;
    }
    return (stage >= 1 && stage <= n) ? t[stage - 1] : 1.0;
}

}  // namespace

std::vector<double> SpeciesHost::thresholds() const {
    std::vector<double> t;
    for (const MetalTr& r : tr) t.push_back(r.eth);
    return t;
}

bool species_build(const mochii_params& p, SpeciesHost& s, std::string* err) {
    static const char* names[11] = {"c", "n", "o", "ne", "s", "ar", "mg", "fe", "si", "cl", "ca"};
    const double ab[11] = {p.abund_C, p.abund_N, p.abund_O, p.abund_Ne, p.abund_S, p.abund_Ar,
                           p.abund_Mg, p.abund_Fe, p.abund_Si, p.abund_Cl, p.abund_Ca};
    const std::string dir = atomic_dir(p);
    s = SpeciesHost();
    std::vector<std::string> table_files;
    for (int k = 0; k < 11; ++k) {
        if (ab[k] <= 0.0) continue;
        ElementFile e;
        if (!parse_element(dir + "/element_" + names[k] + ".txt", e, err)) return false;
        MetalEl m;
        m.Z = e.Z;
        m.nstage = e.nstage;
        m.tr0 = (int)s.tr.size();
        m.st0 = (int)s.st.size();
        m.kind = std::string(names[k]) == "c" ? 1 : std::string(names[k]) == "o" ? 2 : 0;
        m.abund = ab[k];
        const int ie = (int)s.el.size();
        for (int it = 1; it <= e.nstage - 1; ++it) {
            if ((int)s.tr.size() >= kMaxTr) {
                if (err) *err = "active metal transitions exceed the packet-cache capacity (64)";
                return false;
            }
            const int q = it - 1;
            MetalTr r{};
            r.ie = ie;
            r.it = it;
            r.cxi_form = e.cxi_form[q];
            r.cxr_form = e.cxr_form[q];
            r.ndr = e.ndr[q];
            r.has_dr2 = e.has_dr2[q];
            r.has_rr2 = e.has_rr2[q];
            r.eth = e.eth[q];
            r.cidr = dere_ratio(e.Z, it, p.ci_dere_hybrid != 0);
            std::copy(e.ci[q], e.ci[q] + 5, r.ci);
            std::copy(e.rr[q], e.rr[q] + 6, r.rr);
            std::copy(e.dr_c[q], e.dr_c[q] + 9, r.dr_c);
            std::copy(e.dr_e[q], e.dr_e[q] + 9, r.dr_e);
            std::copy(e.dr2[q], e.dr2[q] + 4, r.dr2);
            std::copy(e.rr2[q], e.rr2[q] + 2, r.rr2);
            std::copy(e.cxi[q], e.cxi[q] + 6, r.cxi);
            std::copy(e.cxr[q], e.cxr[q] + 6, r.cxr);
            s.tr.push_back(r);
            s.form.push_back(e.photo_form[q]);
            s.photo.insert(s.photo.end(), e.photo[q], e.photo[q] + 8);
        }
        for (int i = 1; i <= e.nstage; ++i) {
            MetalStage g{};
            g.table = -1;
            std::vector<double> A, Ti;
            const std::string stem = std::string(names[k]) + "_" + std::to_string(i);
            if (cooling_fit_read(dir + "/cooling_" + stem + ".txt", A, Ti)) {
                g.has_cool = 1;
                g.nterm = (int)A.size();
                std::copy(A.begin(), A.end(), g.A);
                std::copy(Ti.begin(), Ti.end(), g.Ti);
                if (p.cooling_local_ne) {
                    const std::string suf = (p.fe_levels_full && std::string(names[k]) == "fe") ? "_full" : "";
                    std::ifstream probe(dir + "/nlevel_" + stem + suf + ".txt");
                    if (probe) {
                        g.table = (int)table_files.size();
                        table_files.push_back(dir + "/nlevel_" + stem + suf + ".txt");
                    }
                }
            }
            s.st.push_back(g);
        }
        s.el.push_back(m);
    }
    // threshold order: stable insertion sort of species_setup (species_mod.f90:207-225)
    const int ntr = (int)s.tr.size();
    std::vector<int> order(ntr);
    for (int j = 0; j < ntr; ++j) order[j] = j;
    for (int i = 1; i < ntr; ++i) {
        const int v = order[i];
        int j = i - 1;
        while (j >= 0 && !(s.tr[order[j]].eth <= s.tr[v].eth)) {
            order[j + 1] = order[j];
            --j;
        }
        order[j + 1] = v;
    }
    std::vector<double> photo_el = s.photo;
    std::vector<int> form_el = s.form;
    s.eth_flat.resize(ntr);
    for (int k = 0; k < ntr; ++k) {
        const int j = order[k];
        s.tr[j].flat = k;
        s.eth_flat[k] = s.tr[j].eth;
        s.form[k] = form_el[j];
        std::copy(photo_el.begin() + 8 * j, photo_el.begin() + 8 * j + 8, s.photo.begin() + 8 * k);
    }
    // n-level tables, one thread per ion (each is an independent set of solves)
    s.ntab = (int)table_files.size();
    std::vector<std::vector<double>> lr(s.ntab), ss(s.ntab);
    std::vector<int> ok(s.ntab, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < s.ntab; ++t)
        pool.emplace_back([&, t] { ok[t] = nlevel_table_build(table_files[t], lr[t], ss[t]) ? 1 : 0; });
    for (auto& th : pool) th.join();
    for (int t = 0; t < s.ntab; ++t)
        if (!ok[t]) {
            if (err) *err = "cannot read the n-level atom " + table_files[t];
            return false;
        }
    s.lamref.resize((size_t)s.ntab * kNlNT);
    s.Ssup.resize((size_t)s.ntab * kNlNT * kNlNNE);
    for (int t = 0; t < s.ntab; ++t) {
        std::copy(lr[t].begin(), lr[t].end(), s.lamref.begin() + (size_t)t * kNlNT);
        std::copy(ss[t].begin(), ss[t].end(), s.Ssup.begin() + (size_t)t * kNlNT * kNlNNE);
    }
    return true;
}

void species_moment_tables(SpeciesHost& s, double emin, double emax) {
    const int ntr = (int)s.tr.size();
    const int ntrp = (ntr + 3) / 4 * 4;
    const double pi = 3.141592653589793;
    auto integrand = [&](int k, int q, double E) {
        const double* c = &s.photo[8 * k];
        const double sk = (s.form[k] == 2 ? sigma_vy95(E, c[0], c[1], c[2], c[3], c[4], c[5], c[6])
                                          : sigma_vfky96(E, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7])) * 1.0e18;
        return q == 0 ? sk / E : sk * std::max(1.0 - s.eth_flat[k] / E, 0.0);
    };
    double node[kMomDeg];
    for (int j = 0; j < kMomDeg; ++j) node[j] = std::cos(pi * (j + 0.5) / kMomDeg);
    // Chebyshev interpolation coefficients of integrand (k, q) on [lo, hi]
    auto coefs = [&](int k, int q, double lo, double hi, double* a) {
        const double mid = 0.5 * (lo + hi), half = 0.5 * (hi - lo);
        double f[kMomDeg];
        for (int j = 0; j < kMomDeg; ++j) f[j] = integrand(k, q, mid + half * node[j]);
        for (int m = 0; m < kMomDeg; ++m) {
            double v = 0.0;
            for (int j = 0; j < kMomDeg; ++j) v += f[j] * std::cos(m * std::acos(node[j]));
            a[m] = v * (m == 0 ? 1.0 : 2.0) / kMomDeg;
        }
    };
    auto bin_error = [&](double lo, double hi) {
        double worst = 0.0;
        const double mid = 0.5 * (lo + hi), half = 0.5 * (hi - lo);
        for (int k = 0; k < ntr; ++k) {
            if (s.eth_flat[k] > lo) continue;
            for (int q = 0; q < 2; ++q) {
                double a[kMomDeg], peak = 0.0, err = 0.0;
                coefs(k, q, lo, hi, a);
                for (int i = 0; i <= 32; ++i) {
                    const double t = -1.0 + 2.0 * i / 32.0;
                    const double ex = integrand(k, q, mid + half * t);
                    double tm1 = 1.0, tm = t, ap = a[0] + a[1] * t;
                    for (int m = 2; m < kMomDeg; ++m) {
                        const double tn = 2.0 * t * tm - tm1;
                        ap += a[m] * tn;
                        tm1 = tm;
                        tm = tn;
                    }
                    peak = std::max(peak, std::fabs(ex));
                    err = std::max(err, std::fabs(ap - ex));
                }
                if (peak > 0.0) worst = std::max(worst, err / peak);
            }
        }
        return worst;
    };
    std::vector<double> bp{emin, emax};
    for (double e : {13.598, 24.587, 54.416}) if (e > emin && e < emax) bp.push_back(e);
    for (double e : s.eth_flat) if (e > emin && e < emax) bp.push_back(e);
    std::sort(bp.begin(), bp.end());
    bp.erase(std::unique(bp.begin(), bp.end()), bp.end());
    std::vector<std::pair<double, double>> todo;
    const double dl = 0.04;
    for (size_t i = 0; i + 1 < bp.size(); ++i) {
        const double lo = bp[i], hi = bp[i + 1];
        const int n = std::max(1, (int)std::ceil(std::log(hi / lo) / dl - 1e-9));
        for (int j = 0; j < n; ++j)
            todo.push_back({j == 0 ? lo : lo * std::exp(std::log(hi / lo) * (double)j / n),
                            j == n - 1 ? hi : lo * std::exp(std::log(hi / lo) * (double)(j + 1) / n)});
    }
    s.medge.clear();
    for (auto& seg : todo) {   // depth-first halving in ln E, in ascending order
        std::vector<std::pair<std::pair<double, double>, int>> st{{seg, 0}};
        while (!st.empty()) {
            const auto cur = st.back();
            st.pop_back();
            const double lo = cur.first.first, hi = cur.first.second;
            if (cur.second < 16 && bin_error(lo, hi) > kMomTol) {
                const double m = std::sqrt(lo * hi);
                st.push_back({{m, hi}, cur.second + 1});
                st.push_back({{lo, m}, cur.second + 1});
            } else {
                s.medge.push_back(lo);
            }
        }
    }
    s.medge.push_back(bp.back());
    const int nmb = (int)s.medge.size() - 1;
    s.mcoef.assign((size_t)nmb * kMomDeg * ntrp * 2, 0.0);
    s.mb0.assign(ntr, nmb);
    for (int k = 0; k < ntr; ++k)
        for (int b = 0; b < nmb; ++b) {
            const double lo = s.medge[b], hi = s.medge[b + 1];
            if (s.eth_flat[k] > lo) continue;   // thresholds are edges: inactive over the whole bin
            s.mb0[k] = std::min(s.mb0[k], b);
            for (int q = 0; q < 2; ++q) {
                double a[kMomDeg];
                coefs(k, q, lo, hi, a);
                for (int m = 0; m < kMomDeg; ++m) s.mcoef[(((size_t)b * kMomDeg + m) * ntrp + k) * 2 + q] = a[m];
            }
        }
}

}  // namespace mochii
