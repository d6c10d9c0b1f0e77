// Oracle C entry points for ctypes (test infrastructure only).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "orc_core.h"
#include "orc_thermal.h"
#include "orc_species.h"
#include "orc_amr.h"

using namespace orc;

namespace {
thread_local std::string g_err;
void copy_err(char* buf, int n) {
    if (buf && n > 0) {
        std::strncpy(buf, g_err.c_str(), (size_t)n - 1);
        buf[n - 1] = 0;
    }
}
}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

// Scrambled uniforms u[i*nd + d] for 0-based indices idx0..idx0+n-1
// (qmc_uniforms_stream, qmc_mod.f90:157-168).
int orc_qmc_uniforms(int seed, int stream, long long idx0, long long n, int nd, double* out) {
    if (nd < 1 || nd > 12 || (stream != 1 && stream != 2)) return 1;
    Qmc q;
    q.setup(seed);
    for (long long i = 0; i < n; ++i)
        for (int d = 1; d <= nd; ++d) out[i * nd + d - 1] = q.uniform(idx0 + i, d, stream);
    return 0;
}

// Unscrambled codes (qmc_uniforms_raw, qmc_mod.f90:174-184).
int orc_qmc_raw_codes(long long idx0, long long n, int nd, unsigned* out) {
    if (nd < 1 || nd > 12) return 1;
    Qmc q;
    q.setup(0);
    for (long long i = 0; i < n; ++i)
        for (int d = 1; d <= nd; ++d) out[i * nd + d - 1] = q.sobol_code(idx0 + i, d);
    return 0;
}

void orc_qmc_keys(int seed, unsigned* out24) {
    Qmc q;
    q.setup(seed);
    for (int s = 0; s < 2; ++s)
        for (int d = 0; d < 12; ++d) out24[s * 12 + d] = q.key[s][d];
}

// ---- samplers ------------------------------------------------------------
void* orc_sampler_planck(double T, double emin, double emax, double rtol, const double* thr, int nthr) {
    auto* s = new Sampler();
    std::vector<double> t(thr, thr + nthr);
    if (!build_planck_sampler(*s, T, emin, emax, rtol, t, &g_err)) {
        delete s;
        return nullptr;
    }
    return s;
}
void* orc_sampler_tab(const double* e, const double* f, int n) {
    auto* s = new Sampler();
    if (!build_tabulated_sampler(*s, std::vector<double>(e, e + n), std::vector<double>(f, f + n), &g_err)) {
        delete s;
        return nullptr;
    }
    return s;
}
void* orc_sampler_tab_band(const double* e, const double* f, int n, double emin, double emax) {
    auto* s = new Sampler();
    if (!build_tabulated_band_sampler(*s, std::vector<double>(e, e + n), std::vector<double>(f, f + n), emin, emax,
                                      &g_err)) {
        delete s;
        return nullptr;
    }
    return s;
}
int orc_sampler_size(void* h) { return (int)static_cast<Sampler*>(h)->energy.size(); }
double orc_sampler_total(void* h) { return static_cast<Sampler*>(h)->total_integral; }
void orc_sampler_get(void* h, double* e, double* f, double* c) {
    auto* s = static_cast<Sampler*>(h);
    for (size_t i = 0; i < s->energy.size(); ++i) {
        e[i] = s->energy[i];
        f[i] = s->density[i];
        c[i] = s->cdf[i];
    }
}
void orc_sampler_sample(void* h, const double* u, long long n, double* out) {
    auto* s = static_cast<Sampler*>(h);
    for (long long i = 0; i < n; ++i) out[i] = sample_energy_cdf(*s, u[i]);
}
void orc_sampler_cdf(void* h, const double* e, long long n, double* out) {
    auto* s = static_cast<Sampler*>(h);
    for (long long i = 0; i < n; ++i) out[i] = energy_cdf_value(*s, e[i]);
}
void orc_sampler_free(void* h) { delete static_cast<Sampler*>(h); }

// ---- scalar physics --------------------------------------------------------
// name in {alphaA_HII, alphaB_HII, alpha1_HII, ... , ci_HI, ci_HeI, ci_HeII,
// sigma_HI, sigma_HeI, sigma_HeII}; model 0 = badnell_milne, 1 = hui_gnedin.
int orc_eval(const char* name, int recomb_model, const double* x, long long n, double* out) {
    RateModel m;
    m.recomb = recomb_model;
    std::string s(name);
    for (long long i = 0; i < n; ++i) {
        const double T = x[i];
        double v;
        if (s == "alphaA_HII") v = alphaA_HII(m, T);
        else if (s == "alphaB_HII") v = alphaB_HII(m, T);
        else if (s == "alpha1_HII") v = alpha1_HII(T);
        else if (s == "alphaA_HeII") v = alphaA_HeII(m, T);
        else if (s == "alphaB_HeII") v = alphaB_HeII(m, T);
        else if (s == "alpha1_HeII") v = alpha1_HeII(T);
        else if (s == "alphaA_HeIII") v = alphaA_HeIII(m, T);
        else if (s == "alphaB_HeIII") v = alphaB_HeIII(m, T);
        else if (s == "alpha1_HeIII") v = alpha1_HeIII(T);
        else if (s == "ci_HI") v = ci_HI(m, T);
        else if (s == "ci_HeI") v = ci_HeI(m, T);
        else if (s == "ci_HeII") v = ci_HeII(m, T);
        else if (s == "sigma_HI") v = sigma_HI(T);
        else if (s == "sigma_HeI") v = sigma_HeI(T);
        else if (s == "sigma_HeII") v = sigma_HeII(T);
        else return 1;
        out[i] = v;
    }
    return 0;
}

// Bin edges for a namelist (ion_setup band part).
int orc_band_edges(const char* nl, double* out, int cap) {
    Par p;
    if (!parse_namelist(nl, p, &g_err)) return -1;
    Band b;
    if (!band_setup(p, b, &g_err)) return -1;
    if ((int)b.eedge.size() > cap) return -1;
    for (size_t i = 0; i < b.eedge.size(); ++i) out[i] = b.eedge[i];
    return (int)b.eedge.size();
}

// ---- simulation ------------------------------------------------------------
void* orc_sim_new(const char* namelist, int nthreads, char* errbuf, int errlen) {
    auto* s = new Sim();
    s->nthreads = nthreads;
    if (!s->setup(namelist, &g_err)) {
        copy_err(errbuf, errlen);
        delete s;
        return nullptr;
    }
    return s;
}
void orc_sim_free(void* h) { delete static_cast<Sim*>(h); }
int orc_sim_nleaf(void* h) { return static_cast<Sim*>(h)->grid.nleaf; }
int orc_sim_nnu(void* h) { return static_cast<Sim*>(h)->band.nnu_band; }
double orc_sim_ion_Ltot(void* h) { return static_cast<Sim*>(h)->band.ion_Ltot; }
void orc_sim_set_nphotons(void* h, long long n) { static_cast<Sim*>(h)->par.nphotons = n; }
int orc_sim_transport_pass(void* h) {
    static_cast<Sim*>(h)->transport_pass();
    return 0;
}
// Each update is followed by gas_opacity_fill, as in the iteration loop of
// main.f90:130-171.
int orc_sim_equilibrium_update(void* h, double* metrics2) {
    auto* s = static_cast<Sim*>(h);
    s->gas_equilibrium_update(&metrics2[0], &metrics2[1]);
    s->opacity_fill();
    return 0;
}
int orc_sim_thermal_update(void* h, double* metrics4) {
    auto* s = static_cast<Sim*>(h);
    if (!s->th) return 1;
    s->gas_thermal_update(metrics4);
    s->opacity_fill();
    return 0;
}
// Metal registry probes for the charge-exchange gates (leaf 0 of the sim,
// whose Gammas are zero before a transport pass).
int orc_sim_metal_nel(void* h) {
    auto* s = static_cast<Sim*>(h);
    return s->metals() ? (int)s->sp->el.size() : 0;
}
int orc_sim_metal_el(void* h, int ie, char* name3, int* Z, int* nstage) {
    auto* s = static_cast<Sim*>(h);
    if (!s->metals() || ie < 0 || ie >= (int)s->sp->el.size()) return -1;
    const Element& e = s->sp->el[ie];
    std::strncpy(name3, e.name.c_str(), 2);
    name3[2] = 0;
    *Z = e.Z;
    *nstage = e.nstage;
    return 0;
}
double orc_sim_metal_eth(void* h, int ie, int it) { return static_cast<Sim*>(h)->sp->el[ie].eth[it - 1]; }
void orc_sim_metal_cx(void* h, int ie, int it, double T, double* out2) {
    const Element& e = static_cast<Sim*>(h)->sp->el[ie];
    out2[0] = e.cxi_form[it - 1] > 0 ? cx_rate(e.cxi_form[it - 1], e.cxi[it - 1], T) : 0.0;
    out2[1] = e.cxr_form[it - 1] > 0 ? cx_rate(e.cxr_form[it - 1], e.cxr[it - 1], T) : 0.0;
}
void orc_sim_metal_sums(void* h, double T, double nH, double ne, double nHI, double nHII, double* out3) {
    auto* s = static_cast<Sim*>(h);
    MetalCache c;
    s->sp->prepare(0, T, s->rm, c);
    s->sp->metal_sums(c, nH, ne, nHI, nHII, out3[0], out3[1], out3[2]);
}
void orc_sim_metal_fractions(void* h, int ie, double T, double ne, double nHI, double nHII, double* out) {
    auto* s = static_cast<Sim*>(h);
    s->sp->fractions(ie, 0, T, ne, nHI, nHII, s->rm, out);
}
// solve_ion_cell on leaf 0 with the sim's metal switches; st4 = x_HI, x_HeI,
// x_HeII in, n_e out.
void orc_sim_solve_cell(void* h, double gH, double gHe1, double gHe2, double nH, double T, int caseA, double* st4) {
    auto* s = static_cast<Sim*>(h);
    solve_ion_cell(s->rm, s->par.He_abund, gH, gHe1, gHe2, nH, T, caseA != 0, st4[0], st4[1], st4[2], st4[3],
                   s->metals() ? s->sp : nullptr, 0, s->par.metal_ne, s->par.charge_exchange == "two_way");
}
// Metal terms of net_rate on leaf il: cool, cool_H, freefree, heat.
int orc_sim_metal_thermal(void* h, int il, double T, double nH, double ne, double xHI, double* out4) {
    auto* s = static_cast<Sim*>(h);
    if (!s->metals() || !s->th) return -1;
    const MetalThermal m = s->sp->thermal(il, T, nH, ne, nH * xHI, nH * (1.0 - xHI), s->rm, s->th->gff);
    out4[0] = m.cool; out4[1] = m.cool_H; out4[2] = m.freefree; out4[3] = m.heat;
    return 0;
}
// net_rate on leaf il at T from the leaf's current state: out = net, x_HI,
// x_HeI, x_HeII, n_e after the cell solve at T.
int orc_sim_net_rate(void* h, int il, double T, double* out5) {
    auto* s = static_cast<Sim*>(h);
    if (!s->th) return -1;
    double xHI = s->st.xHI[il], xHeI = s->st.xHeI[il], xHeII = s->st.xHeII[il], ne = 0.0;
    out5[0] = s->net_rate(il, T, s->par.case_ab == "A", xHI, xHeI, xHeII, ne);
    out5[1] = xHI; out5[2] = xHeI; out5[3] = xHeII; out5[4] = ne;
    return 0;
}
// The thermal bisection on every stride-th leaf with nH > 0, state left
// unchanged (the CPU-baseline sample); returns the leaves solved.
long long orc_sim_thermal_sample(void* h, long long stride) {
    auto* s = static_cast<Sim*>(h);
    if (!s->th || stride < 1) return -1;
    long long solved = 0;
#pragma omp parallel for num_threads(std::max(1, s->nthreads)) schedule(dynamic, 16) reduction(+ : solved)
    for (long long il = 0; il < s->grid.nleaf; il += stride) {
        if (s->st.nH[il] <= 0.0) continue;
        double x, h1, h2, ne;
        s->thermal_cell((int)il, x, h1, h2, ne);
        ++solved;
    }
    return solved;
}
// Metal registry shape: transitions and stages in element order.
int orc_sim_metal_ntr(void* h) {
    auto* s = static_cast<Sim*>(h);
    return s->metals() ? s->sp->ntr : 0;
}
int orc_sim_metal_nstage(void* h) {
    auto* s = static_cast<Sim*>(h);
    if (!s->metals()) return 0;
    int n = 0;
    for (const Element& e : s->sp->el) n += e.nstage;
    return n;
}
// Thermal building blocks for the tests.
void orc_gff_table(double* logT41, double* z164) {
    GffTable t;
    t.build();
    for (int i = 0; i < 41; ++i) {
        logT41[i] = t.logT[i];
        for (int k = 0; k < 4; ++k) z164[i * 4 + k] = t.z[i][k];
    }
}
double orc_cooling_total(void* h, double T, double nH, double ne, double xHI, double xHeI, double xHeII) {
    auto* s = static_cast<Sim*>(h);
    return cooling_total(*s->th, s->rm, s->par.case_ab == "A", s->par.He_abund, T, nH, ne, xHI, xHeI, xHeII);
}
double orc_nlevel_cooling_at(const char* path, double T, double ne) {
    NlevelAtom a;
    if (!a.load(path)) return -1.0;
    return nlevel_cooling_at(a, T, ne);
}
// Philox packet-stream uniforms: out[i] = draw n0 + i of (seed, stream, packet)
void orc_philox(unsigned long long seed, unsigned stream, unsigned long long packet, unsigned n0, int n,
                double* out) {
    for (int i = 0; i < n; ++i) out[i] = philox_uniform(seed, stream, packet, n0 + (unsigned)i);
}
void orc_philox_block(const unsigned* ctr4, const unsigned* key2, unsigned* out4) {
    philox4x32_10(ctr4, key2, out4);
}
// grain optics of the simulation at energies E: (sabs, ssca, g) per energy
int orc_sim_dust_optics(void* h, long long n, const double* E, double* out3) {
    auto* s = static_cast<Sim*>(h);
    if (!s->par.ion_add_dust) return -1;
    for (long long i = 0; i < n; ++i) {
        out3[3 * i] = s->dust.sabs_at(E[i]);
        out3[3 * i + 1] = s->dust.ssca_at(E[i]);
        out3[3 * i + 2] = s->dust.g_at(E[i]);
    }
    return 0;
}
// energy ledger (emitted, absorbed, escaped) and segment counts
void orc_sim_energy(void* h, double* e3, long long* segs2) {
    auto* s = static_cast<Sim*>(h);
    e3[0] = (double)s->tally.emitted;
    e3[1] = (double)s->tally.absorbed;
    e3[2] = (double)s->tally.escaped;
    segs2[0] = s->tally.direct_segments;
    segs2[1] = s->tally.scattered_segments;
}
// slab_Iesc of the last pass (jtally_mod.f90:39-86): n = 2 nmu values,
// [face * nmu + bin], face 0 top; returns the count, 0 without the slab.
int orc_sim_slab(void* h, double* out, int n) {
    auto* s = static_cast<Sim*>(h);
    const int m = (int)s->tally.slab.size();
    for (int k = 0; k < m && k < n; ++k) out[k] = s->tally.slab[k];
    return m;
}
// field names: nH x_HI x_HeI x_HeII n_e T_e gamma_HI gamma_HeI gamma_HeII
// heat_HI heat_HeI heat_HeII jt_ion (nleaf*nnu, leaf-major) hhe (nleaf*6)
long long orc_sim_get(void* h, const char* name, double* out, long long cap) {
    auto* s = static_cast<Sim*>(h);
    std::string n(name);
    const std::vector<double>* v = nullptr;
    if (n == "nH") v = &s->st.nH;
    else if (n == "x_HI") v = &s->st.xHI;
    else if (n == "x_HeI") v = &s->st.xHeI;
    else if (n == "x_HeII") v = &s->st.xHeII;
    else if (n == "n_e") v = &s->st.ne;
    else if (n == "T_e") v = &s->st.Te;
    else if (n == "gamma_HI") v = &s->gamma_HI;
    else if (n == "gamma_HeI") v = &s->gamma_HeI;
    else if (n == "gamma_HeII") v = &s->gamma_HeII;
    else if (n == "heat_HI") v = &s->heat_HI;
    else if (n == "heat_HeI") v = &s->heat_HeI;
    else if (n == "heat_HeII") v = &s->heat_HeII;
    else if (n == "jt_ion") v = &s->tally.jt;
    else if (n == "heat_dust") v = &s->heat_dust;
    else if (n == "g0_fuv") v = &s->g0_fuv;
    else if (n == "rhokap") v = &s->st.rhokap;
    else if (n == "hhe") v = &s->tally.hhe;
    else if (n == "eedge") v = &s->band.eedge;
    else if (s->metals() && (n == "gamma_metal" || n == "heat_metal" || n == "x_metal" || n == "metal_raw")) {
        // leaf-major blocks in element order: (it, il) -> out[il*ntr + j]
        const Species& sp = *s->sp;
        const int nl = sp.nleaf;
        std::vector<double> tmp;
        if (n == "metal_raw") {
            tmp = s->tally.metal;
        } else if (n == "x_metal") {
            int ns = 0;
            for (const Element& e : sp.el) ns += e.nstage;
            tmp.assign((size_t)ns * nl, 0.0);
            int j0 = 0;
            for (size_t ie = 0; ie < sp.el.size(); ++ie) {
                for (int i = 0; i < sp.el[ie].nstage; ++i)
                    for (int il = 0; il < nl; ++il) tmp[(size_t)il * ns + j0 + i] = sp.stage_frac[ie][(size_t)i * nl + il];
                j0 += sp.el[ie].nstage;
            }
        } else {
            const auto& src = n == "gamma_metal" ? sp.egam : sp.eheat;
            tmp.assign((size_t)sp.ntr * nl, 0.0);
            int j0 = 0;
            for (size_t ie = 0; ie < sp.el.size(); ++ie) {
                const int nt = sp.el[ie].nstage - 1;
                for (int i = 0; i < nt; ++i)
                    for (int il = 0; il < nl; ++il) tmp[(size_t)il * sp.ntr + j0 + i] = src[ie][(size_t)i * nl + il];
                j0 += nt;
            }
        }
        if ((long long)tmp.size() > cap) return -(long long)tmp.size();
        std::memcpy(out, tmp.data(), tmp.size() * sizeof(double));
        return (long long)tmp.size();
    }
    if (!v) return -1;
    if ((long long)v->size() > cap) return -(long long)v->size();
    std::memcpy(out, v->data(), v->size() * sizeof(double));
    return (long long)v->size();
}
long long orc_sim_set(void* h, const char* name, const double* in, long long n) {
    auto* s = static_cast<Sim*>(h);
    std::string nm(name);
    std::vector<double>* v = nullptr;
    if (nm == "x_HI") v = &s->st.xHI;
    else if (nm == "x_HeI") v = &s->st.xHeI;
    else if (nm == "x_HeII") v = &s->st.xHeII;
    else if (nm == "n_e") v = &s->st.ne;
    else if (nm == "T_e") v = &s->st.Te;
    else if (nm == "nH") v = &s->st.nH;
    else if (nm == "gamma_HI") v = &s->gamma_HI;
    else if (nm == "gamma_HeI") v = &s->gamma_HeI;
    else if (nm == "gamma_HeII") v = &s->gamma_HeII;
    else if (nm == "heat_HI") v = &s->heat_HI;
    else if (nm == "heat_HeI") v = &s->heat_HeI;
    else if (nm == "heat_HeII") v = &s->heat_HeII;
    else if (nm == "heat_dust") v = &s->heat_dust;
    else if (s->metals() && (nm == "gamma_metal" || nm == "heat_metal")) {
        // leaf-major in element order, in[il*ntr + j], as orc_sim_get returns them
        Species& sp = *s->sp;
        const int nl = sp.nleaf;
        if (n != (long long)sp.ntr * nl) return -1;
        auto& dst = nm == "gamma_metal" ? sp.egam : sp.eheat;
        int j0 = 0;
        for (size_t ie = 0; ie < sp.el.size(); ++ie) {
            const int nt = sp.el[ie].nstage - 1;
            for (int i = 0; i < nt; ++i)
                for (int il = 0; il < nl; ++il) dst[ie][(size_t)i * nl + il] = in[(size_t)il * sp.ntr + j0 + i];
            j0 += nt;
        }
        return n;
    }
    if (!v || (long long)v->size() != n) return -1;
    std::memcpy(v->data(), in, (size_t)n * sizeof(double));
    if (nm.rfind("gamma_", 0) != 0 && nm.rfind("heat_", 0) != 0 && !s->defer_fill)
        s->opacity_fill();   // the stage cache follows the state it is read from
    return n;
}
// Several state fields at once: orc_sim_defer_fill(h, 1), the sets, then
// orc_sim_defer_fill(h, 0) refreshes the opacities once.
void orc_sim_defer_fill(void* h, int on) {
    auto* s = static_cast<Sim*>(h);
    s->defer_fill = on != 0;
    if (!on) s->opacity_fill();
}
// The thermal bisection (thermal_cell, thermal_mod.f90:159-188) of the given
// leaves from the current state and rates, state unchanged: out5[k*5 + .] =
// T_e, x_HI, x_HeI, x_HeII, n_e of leaf idx[k] (as the solve leaves them,
// before under-relaxation).  Returns the leaves solved, -1 without T_e.
long long orc_sim_thermal_cells(void* h, const long long* idx, long long n, double* out5) {
    auto* s = static_cast<Sim*>(h);
    if (!s->th) return -1;
#pragma omp parallel for num_threads(std::max(1, s->nthreads)) schedule(dynamic, 8)
    for (long long k = 0; k < n; ++k) {
        const long long il = idx[k];
        double* o = out5 + 5 * k;
        if (il < 0 || il >= s->grid.nleaf || s->st.nH[il] <= 0.0) {
            o[0] = o[1] = o[2] = o[3] = o[4] = -1.0;
            continue;
        }
        double x, h1, h2, ne;
        o[0] = s->thermal_cell((int)il, x, h1, h2, ne);
        o[1] = x; o[2] = h1; o[3] = h2; o[4] = ne;
    }
    return n;
}
// The imaging pass (ionizing_field_and_rates with with_peel, main.f90:234-235):
// one transport pass that also peels every packet toward the observers.
int orc_sim_transport_pass_peel(void* h) {
    auto* s = static_cast<Sim*>(h);
    if (!s->peel_on) return 1;
    s->peel_pass = true;
    s->transport_pass();
    s->peel_pass = false;
    return 0;
}
// Peel-off images of the last imaging pass, which = 0 direct, 1 scattered,
// 2 unattenuated direct; (nobs, nchan, nyim, nxim) in erg/s per code length^2
// per pixel (before ion_peel_write's conversion).  shape4 receives the shape.
long long orc_sim_peel_image(void* h, int which, double* out, long long cap, int* shape4) {
    auto* s = static_cast<Sim*>(h);
    const std::vector<double>& v = which == 0 ? s->tally.img_dir : which == 1 ? s->tally.img_sca : s->tally.img_dir0;
    shape4[0] = (int)s->obs.size(); shape4[1] = s->nchan; shape4[2] = s->par.nyim; shape4[3] = s->par.nxim;
    if ((long long)v.size() > cap) return -(long long)v.size();
    std::memcpy(out, v.data(), v.size() * sizeof(double));
    return (long long)v.size();
}
// Observer k: x, y, z, alpha, beta, gamma, distance, dxim, dyim, then the
// rotation matrix row by row (18 doubles).
int orc_sim_peel_observer(void* h, int k, double* out18) {
    auto* s = static_cast<Sim*>(h);
    if (k < 0 || k >= (int)s->obs.size()) return 1;
    const PeelObserver& o = s->obs[k];
    const double v[7] = {o.x, o.y, o.z, o.alpha, o.beta, o.gamma, o.distance};
    for (int i = 0; i < 7; ++i) out18[i] = v[i];
    out18[7] = s->dxim; out18[8] = s->dyim;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out18[9 + 3 * i + j] = o.R[i][j];
    return 0;
}
// Diffuse packets launched by the last transport pass (diffuse_nphot).
long long orc_sim_diffuse_count(void* h) { return static_cast<Sim*>(h)->diffuse_nphot; }
// Diffuse field: build from the current state, then launch records.
double orc_sim_diffuse_build(void* h, long long* nphot) {
    auto* s = static_cast<Sim*>(h);
    s->diffuse_build(s->band.ion_Ltot / (double)s->par.nphotons);
    *nphot = s->diffuse_nphot;
    return s->diffuse_lum;
}
void orc_sim_diffuse_photon(void* h, long long ip, double* out8) {
    auto* s = static_cast<Sim*>(h);
    Photon ph;
    s->gen_diffuse_qmc(ip, ph);
    out8[0] = ph.x; out8[1] = ph.y; out8[2] = ph.z;
    out8[3] = ph.kx; out8[4] = ph.ky; out8[5] = ph.kz;
    out8[6] = ph.E; out8[7] = ph.inu;
}
double orc_milne_sample(void* h, int ich, double T, double u) {
    auto* s = static_cast<Sim*>(h);
    return s->milne.sample(ich, T, u, s->par.eion_max);
}
// Launch record of packet ip: x,y,z,kx,ky,kz,E,inu
void orc_sim_photon(void* h, long long ip, double* out8) {
    auto* s = static_cast<Sim*>(h);
    Photon ph;
    s->gen_photon_qmc(ip, ph);
    out8[0] = ph.x; out8[1] = ph.y; out8[2] = ph.z;
    out8[3] = ph.kx; out8[4] = ph.ky; out8[5] = ph.kz;
    out8[6] = ph.E; out8[7] = ph.inu;
}
// Geometry-only leaf sequences for nray rays (x,y,z,kx,ky,kz each).
int orc_sim_walk_leaves(void* h, long long nray, const double* rays, int max_steps, int* leaves, int* nsteps) {
    auto* s = static_cast<Sim*>(h);
    for (long long r = 0; r < nray; ++r) {
        const double* q = rays + 6 * r;
        nsteps[r] = s->amr_walk()
                        ? s->walk_leaves_amr(q[0], q[1], q[2], q[3], q[4], q[5], max_steps, leaves + r * max_steps)
                        : s->walk_leaves_car(q[0], q[1], q[2], q[3], q[4], q[5], max_steps, leaves + r * max_steps);
        for (int k = nsteps[r]; k < max_steps; ++k) leaves[r * max_steps + k] = -1;
    }
    return 0;
}
// Single-cell solve (ion_balance_mod.f90:53-150), H/He path.
void orc_solve_ion_cell(int recomb_model, double yHe, double gH, double gHe1, double gHe2, double nH, double T,
                        int caseA, double* x3, double* ne) {
    RateModel m;
    m.recomb = recomb_model;
    solve_ion_cell(m, yHe, gH, gHe1, gHe2, nH, T, caseA != 0, x3[0], x3[1], x3[2], *ne);
}


// The 1D thermal reference of the G2a gate (check_g2a.py:150-207) with the
// H I line-cooling fit of atomic_dir/cooling_h_1.txt and no n-level
// suppression.  cfg10 = nnu, emin, emax, tstar, lband, nH, yHe, rsph_pc,
// te_min, te_max; out5 = r_pc, x_HI, x_HeI, x_HeII, T_e, each nr long.
int orc_thermal_1d(const char* atomic_dir, const double* cfg10, int nr, int nsweep, double* out5) {
    Thermal th;
    th.gff.build();
    if (!th.hi_fit.load(std::string(atomic_dir) + "/cooling_h_1.txt")) {
        g_err = std::string("cannot open ") + atomic_dir + "/cooling_h_1.txt";
        return 1;
    }
    th.use_hi_table = false;
    Sphere1D s;
    s.nnu = (int)cfg10[0]; s.emin = cfg10[1]; s.emax = cfg10[2]; s.tstar = cfg10[3]; s.lband = cfg10[4];
    s.nH = cfg10[5]; s.yHe = cfg10[6]; s.rsph_pc = cfg10[7]; s.te_min = cfg10[8]; s.te_max = cfg10[9];
    const RateModel rm;
    return thermal_1d(th, rm, s, nr, nsweep, out5, out5 + nr, out5 + 2 * (size_t)nr, out5 + 3 * (size_t)nr,
                      out5 + 4 * (size_t)nr);
}


// The He I two-photon table of the file at path (hei_twophoton_mod.f90):
// out2 = in-band photons and energy [eV] per 2^1S decay; E[k] = the sampled
// energy of u[k].
int orc_hei_2ph(const char* path, double eion_max, const double* u, long long n, double* E, double* out2) {
    HeI2ph h;
    if (!h.setup(path, eion_max)) {
        g_err = std::string("cannot read ") + path;
        return 1;
    }
    out2[0] = h.n_per_decay;
    out2[1] = h.e_per_decay;
    for (long long k = 0; k < n; ++k) E[k] = h.sample(u[k]);
    return 0;
}
// hei_branch_energies (diffuse_mod.f90:308-325) with the table at path:
// out3 = e3s, e1p, e1s [eV per case-B He II recombination].
int orc_hei_branch_energies(const char* path, double T, double xHI, double xHeI, double* out3) {
    HeI2ph h;
    if (!h.setup(path, 100.0)) {
        g_err = std::string("cannot read ") + path;
        return 1;
    }
    hei_branch_energies(h, T, xHI, xHeI, out3[0], out3[1], out3[2]);
    return 0;
}


// dust_temp_compute on the sim's current Heat_dust and rhokap: out[nleaf] =
// T_dust; ir[240] = L_nu at the IR wavelengths, ir[240] = absorbed power
// (dust_ir_write); lam[240] the wavelengths [um].
int orc_sim_dust_temp(void* h, double* out, double* lam, double* ir) {
    auto* s = static_cast<Sim*>(h);
    if (!s->par.ion_add_dust || s->dust.lam.empty()) return 1;
    DustTemp t;
    t.setup(s->dust);
    const int nleaf = s->grid.nleaf;
    std::vector<double> td(nleaf);
    for (int il = 0; il < nleaf; ++il) td[il] = t.solve(s->st.rhokap[il] / s->par.distance2cm, s->heat_dust[il]);
    std::copy(td.begin(), td.end(), out);
    std::fill(ir, ir + DustTemp::NIR + 1, 0.0);
    const double fourpi = 12.566370614359172953850573533118;
    for (int k = 0; k < DustTemp::NIR; ++k) lam[k] = t.lam_ir[k];
    for (int il = 0; il < nleaf; ++il) {
        if (td[il] <= 0.0) continue;
        const double w = 2.0 * s->grid.lhalf[il] * s->par.distance2cm;
        const double vol = w * w * w, kd = s->st.rhokap[il] / s->par.distance2cm;
        ir[DustTemp::NIR] += s->heat_dust[il] * vol;
        for (int k = 0; k < DustTemp::NIR; ++k) {
            const double nu = 2.99792458e10 / (t.lam_ir[k] * 1.0e-4);
            ir[k] += fourpi * kd * t.sabs_ir[k] * planck_nu(nu, td[il]) * vol;
        }
    }
    return 0;
}


// amr_refine_front on the leaf list in_list with state st6 (6 x nleaf:
// nH, x_HI, x_HeI, x_HeII, n_e, T_e) and rhokap rk (NULL: none): the new
// leaf list in the library's refined-list format (%.17g; x y z level nH
// x_HI x_HeI x_HeII n_e T_e rhokap) to out_list; counts2 = new leaves,
// front leaves; *worst = largest relative change of a conserved integral.
int orc_refine_plan(const char* in_list, const double* st6, const double* rk, double yHe, double te_min, int lbase,
                    int lmax, double eps, double dx, const char* out_list, long long* counts2, double* worst) {
    std::vector<double> x, y, z, nH;
    std::vector<int> lev;
    double boxlen = 0.0;
    if (!read_leaf_list(in_list, x, y, z, lev, nH, &boxlen, &g_err)) return 1;
    Octree o;
    o.build(x, y, z, lev, 0.5 * boxlen);
    const size_t n = x.size();
    std::vector<double> st[6];
    for (int k = 0; k < 6; ++k) st[k].assign(st6 + k * n, st6 + (k + 1) * n);
    std::vector<double> r_k;
    if (rk) r_k.assign(rk, rk + n);
    RefineResult r;
    if (!refine_front(o, st, r_k, yHe, te_min, lbase, lmax, eps, dx, r, &g_err)) return 2;
    FILE* f = std::fopen(out_list, "w");
    if (!f) return 3;
    std::fprintf(f, "%zu %.17g\n", r.x.size(), boxlen);
    for (size_t i = 0; i < r.x.size(); ++i)
        std::fprintf(f, "%.17g %.17g %.17g %d %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", r.x[i], r.y[i], r.z[i],
                     r.lev[i], r.nH[i], r.x1[i], r.x2[i], r.x3[i], r.ne[i], r.te[i], r.rk[i]);
    std::fclose(f);
    counts2[0] = (long long)r.x.size();
    counts2[1] = r.nfront;
    *worst = r.worst;
    return 0;
}

}  // extern "C"
