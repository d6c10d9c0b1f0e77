// Oracle (test infrastructure only): restatement of species_mod.f90 and of the
// metal parts of ion_balance_mod.f90 / thermal_mod.f90, in FP64 with the
// reference's operation order.
#include "orc_species.h"

#include <cmath>
#include <fstream>
#include <sstream>

namespace orc {

// read_element, species_mod.f90:358-423: keyword lines ELEMENT, TRANSITION,
// ETH, PHOTO, PHOTO2, CI, RR, DR, DR2, RR2, CXI, CXR; '#' comments.
static bool read_element(const std::string& path, Element& e) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    int it = 0;
    while (std::getline(f, line)) {
        const size_t a = line.find_first_not_of(" \t");
        if (a == std::string::npos || line[a] == '#') continue;
        std::istringstream s(line.substr(a));
        std::string key;
        s >> key;
        if (key == "ELEMENT") {
            s >> e.name >> e.Z >> e.nstage;
            continue;
        }
        if (key == "TRANSITION") {
            s >> it;
            continue;
        }
        if (it < 1 || it > MAX_ST) continue;
        const int k = it - 1;
        if (key == "ETH") {
            s >> e.eth[k];
        } else if (key == "PHOTO") {
            for (int j = 0; j < 8; ++j) s >> e.photo[k][j];
            e.photo_form[k] = 1;
        } else if (key == "PHOTO2") {
            for (int j = 0; j < 7; ++j) s >> e.photo[k][j];
            e.photo_form[k] = 2;
        } else if (key == "CI") {
            for (int j = 0; j < 5; ++j) s >> e.ci[k][j];
        } else if (key == "RR") {
            for (int j = 0; j < 6; ++j) s >> e.rr[k][j];
        } else if (key == "DR") {
            int n = 0;
            s >> n;
            e.ndr[k] = n;
            for (int j = 0; j < n; ++j) s >> e.dr_c[k][j];
            for (int j = 0; j < n; ++j) s >> e.dr_e[k][j];
        } else if (key == "DR2") {
            for (int j = 0; j < 4; ++j) s >> e.dr2[k][j];
            e.has_dr2[k] = true;
        } else if (key == "RR2") {
            for (int j = 0; j < 2; ++j) s >> e.rr2[k][j];
            e.has_rr2[k] = true;
        } else if (key == "CXI") {
            s >> e.cxi_form[k];
            if (e.cxi_form[k] > 0)
                for (int j = 0; j < 6; ++j) s >> e.cxi[k][j];
        } else if (key == "CXR") {
            s >> e.cxr_form[k];
            if (e.cxr_form[k] > 0)
                for (int j = 0; j < 6; ++j) s >> e.cxr[k][j];
        }
    }
    return e.nstage > 0;
}

static std::string atomic_dir_of(const Par& p) {
    if (!p.atomic_dir.empty()) return p.atomic_dir;
    if (!p.data_dir.empty()) return p.data_dir + "/atomic";
    return "data/atomic";
}

bool Species::setup(const Par& p, int nl, std::string* err) {
    static const char* names[11] = {"c", "n", "o", "ne", "s", "ar", "mg", "fe", "si", "cl", "ca"};
    const double ab[11] = {p.abund_C, p.abund_N, p.abund_O, p.abund_Ne, p.abund_S, p.abund_Ar,
                           p.abund_Mg, p.abund_Fe, p.abund_Si, p.abund_Cl, p.abund_Ca};
    const std::string dir = atomic_dir_of(p);
    nleaf = nl;
    el.clear();
    for (int k = 0; k < 11; ++k) {
        if (ab[k] <= 0.0) continue;
        Element e;
        if (!read_element(dir + "/element_" + names[k] + ".txt", e)) {
            if (err) *err = "cannot open " + dir + "/element_" + names[k] + ".txt";
            return false;
        }
        e.abund = ab[k];
        for (int i = 1; i <= e.nstage; ++i) {
            const std::string f = dir + "/cooling_" + names[k] + "_" + std::to_string(i) + ".txt";
            if (!e.cool[i - 1].load(f)) continue;
            e.has_cool[i - 1] = true;
            if (p.cooling_model == "local_ne") {   // nlevel_cooling_add, nlevel_cooling_mod.f90:104-163
                const std::string suf = (p.fe_levels_full && std::string(names[k]) == "fe") ? "_full" : "";
                NlevelAtom atom;
                if (atom.load(dir + "/nlevel_" + names[k] + "_" + std::to_string(i) + suf + ".txt")) {
                    e.table[i - 1].build(atom);
                    e.has_table[i - 1] = true;
                }
            }
        }
        el.push_back(e);
    }
    ntr = 0;
    for (int ie = 0; ie < (int)el.size(); ++ie)
        for (int i = 1; i <= el[ie].nstage - 1; ++i) {
            if (ntr >= MAX_TR) {
                if (err) *err = "active metal transitions exceed packet-cache capacity 64";
                return false;
            }
            flat_ie[ntr] = ie;
            flat_it[ntr] = i;
            flat_eth[ntr] = el[ie].eth[i - 1];
            ++ntr;
        }
    for (int i = 1; i < ntr; ++i) {   // stable insertion sort by threshold, :209-225
        const int a = flat_ie[i], b = flat_it[i];
        const double t = flat_eth[i];
        int j = i - 1;
        while (j >= 0 && !(flat_eth[j] <= t)) {
            flat_ie[j + 1] = flat_ie[j];
            flat_it[j + 1] = flat_it[j];
            flat_eth[j + 1] = flat_eth[j];
            --j;
        }
        flat_ie[j + 1] = a;
        flat_it[j + 1] = b;
        flat_eth[j + 1] = t;
    }
    for (int k = 0; k < ntr; ++k) flat_of[flat_ie[k]][flat_it[k] - 1] = k;
    egam.assign(el.size(), {});
    eheat.assign(el.size(), {});
    stage_frac.assign(el.size(), {});
    for (size_t ie = 0; ie < el.size(); ++ie) {
        egam[ie].assign((size_t)(el[ie].nstage - 1) * nl, 0.0);
        eheat[ie].assign((size_t)(el[ie].nstage - 1) * nl, 0.0);
        stage_frac[ie].assign((size_t)el[ie].nstage * nl, 0.0);
    }
    return true;
}

std::vector<double> Species::thresholds() const {
    std::vector<double> t;
    for (const Element& e : el)
        for (int it = 1; it <= e.nstage - 1; ++it) t.push_back(e.eth[it - 1]);
    return t;
}

double Species::sigma(int ie, int it, double E) const {
    const double* c = el[ie].photo[it - 1];
    if (el[ie].photo_form[it - 1] == 2) return sigma_vy95(E, c[0], c[1], c[2], c[3], c[4], c[5], c[6]);
    return sigma_vfky96(E, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7]);
}

int Species::packet_sigma(double E, double* sig) const {
    int n = 0;
    for (int k = 0; k < ntr; ++k) {
        if (E < flat_eth[k]) break;
        sig[k] = sigma(flat_ie[k], flat_it[k], E);
        n = k + 1;
    }
    return n;
}

double Species::cached_opacity(const double* sig, int n, int il) const {
    double o = 0.0;
    for (int k = 0; k < n; ++k) {
        const int ie = flat_ie[k], it = flat_it[k];
        o = o + el[ie].abund * stage_frac[ie][(size_t)(it - 1) * nleaf + il] * sig[k];
    }
    return o;
}

void Species::score(double E, const double* sig, int n, int il, double path_lum, double* raw) const {
    for (int k = 0; k < n; ++k) {
        const int ie = flat_ie[k], it = flat_it[k];
        double* r = raw + ((size_t)il * ntr + k) * 2;
        r[0] = r[0] + path_lum * sig[k] / (E * EV2ERG);
        r[1] = r[1] + path_lum * sig[k] * std::max(1.0 - el[ie].eth[it - 1] / E, 0.0);
    }
}

void Species::gamma_compute(const std::vector<double>& raw, const std::vector<double>& fac) {
    for (int ie = 0; ie < (int)el.size(); ++ie)
        for (int it = 1; it <= el[ie].nstage - 1; ++it) {
            const int k = flat_of[ie][it - 1];
            for (int il = 0; il < nleaf; ++il) {
                egam[ie][(size_t)(it - 1) * nleaf + il] = raw[((size_t)il * ntr + k) * 2 + 0] * fac[il];
                eheat[ie][(size_t)(it - 1) * nleaf + il] = raw[((size_t)il * ntr + k) * 2 + 1] * fac[il];
            }
        }
}

double Species::alpha_rec(const Element& e, int it, double T) const {
    const int k = it - 1;
    double a;
    if (e.has_rr2[k]) {
        a = e.rr2[k][0] * std::pow(T / 1.0e4, -e.rr2[k][1]);
    } else {
        const double s0 = std::sqrt(T / e.rr[k][2]), s1 = std::sqrt(T / e.rr[k][3]);
        const double b = e.rr[k][1] + e.rr[k][4] * std::exp(-e.rr[k][5] / T);
        a = e.rr[k][0] / (s0 * std::pow(1.0 + s0, 1.0 - b) * std::pow(1.0 + s1, 1.0 + b));
    }
    for (int j = 0; j < e.ndr[k]; ++j) a = a + std::pow(T, -1.5) * e.dr_c[k][j] * std::exp(-e.dr_e[k][j] / T);
    if (e.has_dr2[k])
        a = a + e.dr2[k][0] * std::pow(T, -1.5) * std::exp(-e.dr2[k][2] / T) *
                    (1.0 + e.dr2[k][1] * std::exp(-e.dr2[k][3] / T));
    return a;
}

double cx_rate(int form, const double* c, double T) {
    double t4 = T / 1.0e4, k, lnT;
    switch (form) {
        case 1:
            k = c[0] * std::pow(T / 300.0, c[1]);
            if (c[2] != 0.0) k = k * std::exp(-c[2] / t4);
            return k;
        case 2:
            return c[0] * std::pow(t4, c[1]) + c[2] * std::pow(t4, c[3]);
        case 3:
            return (c[0] * std::pow(t4, c[1]) + c[2] * std::pow(t4, c[3])) * std::exp(-c[4] / T);
        case 4:
            lnT = std::log(T);
            return std::exp(c[0] + lnT * (c[1] + lnT * (c[2] + lnT * (c[3] + lnT * c[4]))));
        case 5:
            lnT = std::log(T);
            return std::exp(c[0] + lnT * (c[1] + lnT * (c[2] + lnT * (c[3] + lnT * c[4]))) - c[5] / t4);
        case 6:
            t4 = std::min(std::max(t4, 0.5), 5.0);
            k = c[0] * std::pow(t4, c[1]) * (1.0 + c[2] * std::exp(c[3] * t4));
            return std::max(k, 0.0);
        case 7:
            t4 = std::min(std::max(t4, 0.5), 5.0);
            k = c[0] * std::pow(t4, c[1]) * (1.0 + c[2] * std::exp(c[3] * t4)) * std::exp(-c[4] / t4);
            return std::max(k, 0.0);
        default:
            return 0.0;
    }
}

double voronov_ci(const double* c, double T) {
    const double U = c[0] * EV2ERG / (KBOLTZ_CGS * T);
    return c[2] * (1.0 + c[1] * std::sqrt(U)) * std::pow(U, c[4]) * std::exp(-U) / (c[3] + U);
}

void Species::prepare(int il, double T, const RateModel& rm, MetalCache& c) const {
    for (int ie = 0; ie < (int)el.size(); ++ie) {
        const Element& e = el[ie];
        for (int it = 1; it <= e.nstage - 1; ++it) {
            const int k = it - 1;
            c.gam[k][ie] = egam[ie][(size_t)k * nleaf + il];
            c.ci[k][ie] = voronov_ci(e.ci[k], T) * ci_dere_ratio(rm, e.Z, it);
            c.rec[k][ie] = alpha_rec(e, it, T);
            c.cxi[k][ie] = 0.0;
            c.cxr[k][ie] = 0.0;
            if (e.cxi_form[k] > 0) c.cxi[k][ie] = cx_rate(e.cxi_form[k], e.cxi[k], T);
            if (e.cxr_form[k] > 0) c.cxr[k][ie] = cx_rate(e.cxr_form[k], e.cxr[k], T);
        }
    }
}

void Species::metal_sums(const MetalCache& c, double nH, double ne, double nHI, double nHII, double& nem,
                         double& rin, double& rout) const {
    nem = 0.0;
    rin = 0.0;
    rout = 0.0;
    double r[MAX_ST];
    for (int ie = 0; ie < (int)el.size(); ++ie) {
        const int ns = el[ie].nstage;
        for (int it = 1; it <= ns - 1; ++it) {
            const int k = it - 1;
            double rion = c.gam[k][ie] + ne * c.ci[k][ie];
            if (c.cxi[k][ie] > 0.0) rion = rion + nHII * c.cxi[k][ie];
            double rrec = ne * c.rec[k][ie];
            if (c.cxr[k][ie] > 0.0) rrec = rrec + nHI * c.cxr[k][ie];
            r[k] = rion / std::max(rrec, TINEST);
        }
        double s = 1.0, prod = 1.0;
        for (int i = 1; i <= ns - 1; ++i) {
            prod = prod * r[i - 1];
            s = s + prod;
        }
        const double nX = el[ie].abund * nH;
        double fr = 1.0 / s;
        if (ns > 1) rin = rin + c.cxi[0][ie] * nX * fr;
        for (int i = 2; i <= ns; ++i) {
            fr = fr * r[i - 2];
            nem = nem + el[ie].abund * nH * fr * (double)(i - 1);
            rout = rout + c.cxr[i - 2][ie] * nX * fr;
            if (i < ns) rin = rin + c.cxi[i - 1][ie] * nX * fr;
        }
    }
}

void Species::fractions(int ie, int il, double T, double ne, double nHI, double nHII, const RateModel& rm,
                        double* frac) const {
    const Element& e = el[ie];
    const int ns = e.nstage;
    double r[MAX_ST];
    for (int it = 1; it <= ns - 1; ++it) {
        const int k = it - 1;
        double rion = egam[ie][(size_t)k * nleaf + il] + ne * voronov_ci(e.ci[k], T) * ci_dere_ratio(rm, e.Z, it);
        if (e.cxi_form[k] > 0) rion = rion + nHII * cx_rate(e.cxi_form[k], e.cxi[k], T);
        double rrec = ne * alpha_rec(e, it, T);
        if (e.cxr_form[k] > 0) rrec = rrec + nHI * cx_rate(e.cxr_form[k], e.cxr[k], T);
        r[k] = rion / std::max(rrec, TINEST);
    }
    double s = 1.0, prod = 1.0;
    for (int i = 1; i <= ns - 1; ++i) {
        prod = prod * r[i - 1];
        s = s + prod;
    }
    frac[0] = 1.0 / s;
    for (int i = 2; i <= ns; ++i) frac[i - 1] = frac[i - 2] * r[i - 2];
}

void Species::stage_cache_refresh(const State& st, const RateModel& rm) {
    double frac[MAX_ST];
    for (int ie = 0; ie < (int)el.size(); ++ie)
        for (int il = 0; il < nleaf; ++il) {
            const double nHI = st.nH[il] * st.xHI[il];
            const double nHII = st.nH[il] * (1.0 - st.xHI[il]);
            fractions(ie, il, st.Te[il], st.ne[il], nHI, nHII, rm, frac);
            for (int i = 1; i <= el[ie].nstage; ++i) stage_frac[ie][(size_t)(i - 1) * nleaf + il] = frac[i - 1];
        }
}

MetalThermal Species::thermal(int il, double T, double nH, double ne, double nHI, double nHII, const RateModel& rm,
                              const GffTable& gff) const {
    const double kb = 1.380649e-16;
    const double A_CII = 2.321e-6, A_OI = 8.865e-5;
    MetalThermal m;
    double ff = 0.0;
    double frac[MAX_ST];
    for (int ie = 0; ie < (int)el.size(); ++ie) {
        const Element& e = el[ie];
        // one evaluation of the chain serves the four terms: species_fractions
        // is a pure function of (ie, il, T, ne, nHI, nHII)
        fractions(ie, il, T, ne, nHI, nHII, rm, frac);
        const double nel = e.abund * nH;
        for (int i = 1; i <= e.nstage; ++i) {     // metal_cooling
            if (!e.has_cool[i - 1]) continue;
            const double fit = e.cool[i - 1].eval(T);
            const double lam = e.has_table[i - 1] ? e.table[i - 1].apply(fit, T, ne) : fit;
            m.cool = m.cool + ne * nel * frac[i - 1] * lam;
        }
        if (e.name == "c" && e.nstage >= 2) {   // metal_cooling_H, [C II] 158 um
            const double nion = e.abund * nH * frac[1];
            const double qul = 7.6e-10 * std::pow(T / 100.0, 0.14);
            const double qlu = 2.0 * qul * std::exp(-91.25 / T);
            m.cool_H = m.cool_H + nion * nHI * qlu * (91.25 * kb) / (1.0 + nHI * (qul + qlu) / A_CII);
        } else if (e.name == "o") {              // [O I] 63 um
            const double nion = e.abund * nH * frac[0];
            const double qul = 9.2e-11 * std::pow(T / 100.0, 0.67);
            const double qlu = 0.6 * qul * std::exp(-227.7 / T);
            m.cool_H = m.cool_H + nion * nHI * qlu * (227.7 * kb) / (1.0 + nHI * (qul + qlu) / A_OI);
        }
        for (int j = 2; j <= e.nstage; ++j) {     // metal_freefree
            const int zion = j - 1;
            ff = ff + e.abund * frac[j - 1] * (double)(zion * zion) * gff.gbar(T, zion);
        }
        for (int i = 1; i <= e.nstage - 1; ++i)   // metal_heating
            m.heat = m.heat + e.abund * nH * frac[i - 1] * eheat[ie][(size_t)(i - 1) * nleaf + il];
    }
    m.freefree = 1.42554e-27 * std::sqrt(T) * ne * nH * ff;
    return m;
}

double hydrogen_neutral_fraction(const Species& sp, const MetalCache& c, double nH, double ne, double A, double B) {
    double nem, rin, rout;
    double xa = 0.0;
    sp.metal_sums(c, nH, ne, 0.0, nH, nem, rin, rout);
    double Ra = -(A + rin);
    double xb = 1.0;
    sp.metal_sums(c, nH, ne, nH, 0.0, nem, rin, rout);
    double Rb = B + rout;
    const double scale = A + B + std::fabs(Ra) + std::fabs(Rb);
    double x = xb;
    for (int k = 1; k <= 80; ++k) {
        if (Rb == Ra) break;
        x = xb - Rb * (xb - xa) / (Rb - Ra);
        x = std::min(std::max(x, std::min(xa, xb)), std::max(xa, xb));
        sp.metal_sums(c, nH, ne, nH * x, nH * (1.0 - x), nem, rin, rout);
        const double Rx = x * (B + rin + rout) - (A + rin);
        if (std::fabs(Rx) <= 1.0e-15 * scale) break;
        if (std::fabs(xb - xa) <= 1.0e-15) break;
        if (Rx * Rb < 0.0) {
            xa = xb;
            Ra = Rb;
        } else {
            Ra = 0.5 * Ra;
        }
        xb = x;
        Rb = Rx;
    }
    return x;
}

double charge_neutrality_ne(const Species& sp, const RateModel& rm, int il, double T, double nH, double ne_HHe,
                            double xHI, double ne_seed) {
    MetalCache c;
    sp.prepare(il, T, rm, c);
    const double nHI = nH * xHI, nHII = nH * (1.0 - xHI);
    double ne = std::max(ne_seed, 1.0e-12 * nH);
    for (int it = 1; it <= 200; ++it) {
        const double ne_old = ne;
        double nem, rin, rout;
        sp.metal_sums(c, nH, ne_old, nHI, nHII, nem, rin, rout);
        ne = ne_HHe + nem;
        ne = std::max(0.5 * (ne + ne_old), 1.0e-12 * nH);
        if (std::fabs(ne - ne_old) <= 1.0e-10 * ne) break;
    }
    return ne;
}

}  // namespace orc
