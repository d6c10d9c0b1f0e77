// Host-side band and sampler set-up.  See band.h.
#include "band.h"

#include <algorithm>
#include <cmath>

#include "physics.cuh"

namespace mochii {

namespace {
bool fail(std::string* err, const char* m) {
    if (err) *err = m;
    return false;
}

// Planck energy-luminosity shape E^3/(e^x - 1), x = E/kT, with the small-x
// series and the large-x exponential (energy_sampler_mod.f90:277-290).
double planck_shape(double e, double T) {
    const double x = e / (kKbEv * T);
    const double e3 = e * e * e;
    if (x <= 0.0) return 0.0;
    if (x < 1.0e-3) return e3 / (x * (1.0 + 0.5 * x + x * x / 6.0));
    if (x < 700.0) return e3 / (std::exp(x) - 1.0);
    return e3 * std::exp(-x);
}

// Adaptive knot placement: bisect [e0,e1] until the Simpson-vs-trapezoid
// error estimate falls within tol*(|fine| + scale*(e1-e0)/span), depth <= 50
// (energy_sampler_mod.f90:159-185).  Knots are appended left to right.
struct PlanckRefiner {
    double T, tol, scale, span;
    std::vector<double>* e;
    std::vector<double>* f;
    bool refine(double e0, double e1, double f0, double f1, int depth) {
        const double em = 0.5 * (e0 + e1);
        const double fm = planck_shape(em, T);
        const double coarse = 0.5 * (f0 + f1) * (e1 - e0);
        const double fine = 0.25 * (f0 + 2.0 * fm + f1) * (e1 - e0);
        const double est = std::fabs(fine - coarse) / 3.0;
        if (est <= tol * (std::fabs(fine) + scale * (e1 - e0) / span) || depth >= 50) {
            if (e->size() + 1 > 200000) return false;   // MAX_PLANCK_KNOTS
            e->push_back(e1);
            f->push_back(f1);
            return true;
        }
        return refine(e0, em, f0, fm, depth + 1) && refine(em, e1, fm, f1, depth + 1);
    }
};
}  // namespace

// build_tabulated_sampler, energy_sampler_mod.f90:34-64: trapezoid CDF
// normalised to 1 with the last entry pinned to exactly 1.
bool table_from_points(EnergyTable& t, const std::vector<double>& e, const std::vector<double>& f,
                       std::string* err) {
    const size_t n = e.size();
    if (n < 2 || f.size() != n) return fail(err, "energy sampler: table needs at least two matching columns");
    for (size_t i = 0; i < n; ++i)
        if (f[i] < 0.0) return fail(err, "energy sampler: negative spectral density");
    for (size_t i = 1; i < n; ++i)
        if (e[i] <= e[i - 1]) return fail(err, "energy sampler: energies must be strictly ascending");
    t.energy = e;
    t.density = f;
    t.cdf.assign(n, 0.0);
    for (size_t i = 1; i < n; ++i) t.cdf[i] = t.cdf[i - 1] + 0.5 * (f[i - 1] + f[i]) * (e[i] - e[i - 1]);
    t.total = t.cdf[n - 1];
    if (t.total <= 0.0) return fail(err, "energy sampler: zero integrated luminosity");
    for (auto& c : t.cdf) c = c / t.total;
    t.cdf[n - 1] = 1.0;
    return true;
}

// build_planck_sampler, energy_sampler_mod.f90:106-157: mandatory knots at
// the band ends and at every threshold strictly inside it, each interval
// refined adaptively against a 256-panel trapezoid estimate of the band.
bool planck_table(EnergyTable& t, double T, double emin, double emax, double rtol,
                  const std::vector<double>& knots, std::string* err) {
    if (T <= 0.0 || emin < 0.0 || emax <= emin)
        return fail(err, "energy sampler: invalid Planck temperature or energy band");
    if (rtol <= 0.0) return fail(err, "energy sampler: Planck rtol must be positive");
    std::vector<double> m{emin, emax};
    for (double k : knots)
        if (k > emin && k < emax) m.push_back(k);
    std::sort(m.begin(), m.end());
    m.erase(std::unique(m.begin(), m.end()), m.end());
    double scale = 0.0;
    for (int i = 1; i <= 256; ++i) {
        const double e0 = emin + (emax - emin) * (double)(i - 1) / 256.0;
        const double e1 = emin + (emax - emin) * (double)i / 256.0;
        scale = scale + 0.5 * (planck_shape(e0, T) + planck_shape(e1, T)) * (e1 - e0);
    }
    if (scale <= 0.0) return fail(err, "energy sampler: zero Planck band luminosity");
    std::vector<double> e{m[0]}, f{planck_shape(m[0], T)};
    e.reserve(16384);
    f.reserve(16384);
    PlanckRefiner r{T, rtol, scale, emax - emin, &e, &f};
    for (size_t i = 0; i + 1 < m.size(); ++i)
        if (!r.refine(m[i], m[i + 1], planck_shape(m[i], T), planck_shape(m[i + 1], T), 0))
            return fail(err, "energy sampler: Planck knot limit");
    return table_from_points(t, e, f, err);
}

// sample_energy_cdf, energy_sampler_mod.f90:187-238 (host copy; the device
// copy lives in the transport kernel).
double table_sample(const EnergyTable& t, double u) {
    const int n = (int)t.cdf.size();
    const double q = std::min(std::max(u, 0.0), 1.0);
    if (q <= 0.0) return t.energy[0];
    if (q >= 1.0) return t.energy[n - 1];
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi + 2) / 2 - 1;
        if (t.cdf[mid] <= q) lo = mid; else hi = mid;
    }
    const double area = t.cdf[hi] - t.cdf[lo];
    if (area <= 0.0) return t.energy[hi];
    const double dx = t.energy[hi] - t.energy[lo];
    const double y0 = t.density[lo], y1 = t.density[hi];
    const double a = (q - t.cdf[lo]) / area * (0.5 * (y0 + y1) * dx);
    const double slope = (y1 - y0) / dx;
    const double sc = std::max(std::max(std::fabs(y0), std::fabs(y1)), kTinest);
    double off;
    if (std::fabs(slope * dx) <= 64.0 * 2.220446049250313e-16 * sc)
        off = y0 > 0.0 ? a / y0 : 0.0;
    else
        off = 2.0 * a / (y0 + std::sqrt(std::max(0.0, y0 * y0 + 2.0 * slope * a)));
    return t.energy[lo] + std::min(std::max(off, 0.0), dx);
}

// energy_cdf_value, energy_sampler_mod.f90:240-275.
double table_cdf(const EnergyTable& t, double e) {
    const int n = (int)t.energy.size();
    if (e <= t.energy[0]) return 0.0;
    if (e >= t.energy[n - 1]) return 1.0;
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi + 2) / 2 - 1;
        if (t.energy[mid] <= e) lo = mid; else hi = mid;
    }
    const double dx = t.energy[hi] - t.energy[lo];
    const double off = e - t.energy[lo];
    const double y0 = t.density[lo];
    const double slope = (t.density[hi] - y0) / dx;
    const double tot = 0.5 * (y0 + t.density[hi]) * dx;
    const double part = y0 * off + 0.5 * slope * off * off;
    return tot > 0.0 ? t.cdf[lo] + (t.cdf[hi] - t.cdf[lo]) * part / tot : t.cdf[lo];
}

namespace {
// Threshold-aligned ionising edges (build_aligned_edges,
// ion_band_mod.f90:1053-1214): every H/He (priority) and metal threshold
// strictly inside (lo,hi) becomes an edge; near-coincident thresholds
// (|ln ratio| < 0.01) merge, metals give way to H/He; surplus metal
// thresholds are dropped when bins run short; the nion bins are shared
// over the sub-segments by log width with a floor of one (Hamilton
// largest-remainder), each sub-segment log-uniform.
bool aligned_edges(std::vector<double>& edge, int nfuv, int nnu, double lo, double hi,
                   const std::vector<double>& metal, std::string* err) {
    const int nion = nnu - nfuv;
    struct Thr { double e; int pri; };
    std::vector<Thr> c;
    for (double e : {kEthHI, kEthHeI, kEthHeII})
        if (e > lo && e < hi) c.push_back({e, 1});
    for (double e : metal)
        if (e > 0.0 && e > lo && e < hi) c.push_back({e, 0});
    std::stable_sort(c.begin(), c.end(), [](const Thr& a, const Thr& b) { return a.e < b.e; });
    std::vector<Thr> t;
    for (const Thr& x : c) {
        if (!t.empty() && std::fabs(std::log(x.e / t.back().e)) < 0.01) {
            if (x.pri > t.back().pri) t.back() = x;
        } else {
            t.push_back(x);
        }
    }
    while ((int)t.size() + 1 > nion) {
        int best = -1;
        double gap = 1.0e30;
        for (int i = 0; i < (int)t.size(); ++i) {
            if (t[i].pri != 0) continue;
            double g = std::log(t[i].e / (i == 0 ? lo : t[i - 1].e));
            g = std::min(g, std::log((i + 1 == (int)t.size() ? hi : t[i + 1].e) / t[i].e));
            if (g < gap) { gap = g; best = i; }
        }
        if (best < 0) break;
        t.erase(t.begin() + best);
    }
    std::vector<double> pts{lo};
    for (const Thr& x : t) pts.push_back(x.e);
    pts.push_back(hi);
    const int nseg = (int)pts.size() - 1;
    if (nion < nseg) return fail(err, "ion_align_edges: nnu_ion cannot fit the H/He thresholds");
    std::vector<double> w(nseg);
    double wsum = 0.0;
    for (int j = 0; j < nseg; ++j) { w[j] = std::log(pts[j + 1]) - std::log(pts[j]); wsum = wsum + w[j]; }
    std::vector<int> nb(nseg);
    int ntot = 0;
    for (int j = 0; j < nseg; ++j) { nb[j] = std::max(1, (int)((double)nion * w[j] / wsum)); ntot += nb[j]; }
    for (int r = nion - ntot; r > 0; --r) {
        int best = 0;
        double fr = -1.0;
        for (int j = 0; j < nseg; ++j) {
            const double x = (double)nion * w[j] / wsum - (double)nb[j];
            if (x > fr) { fr = x; best = j; }
        }
        ++nb[best];
        ntot++;
    }
    while (ntot > nion) {
        int best = -1;
        double fr = -1.0e30;
        for (int j = 0; j < nseg; ++j) {
            if (nb[j] <= 1) continue;
            const double x = (double)nb[j] - (double)nion * w[j] / wsum;
            if (x > fr) { fr = x; best = j; }
        }
        if (best < 0) break;
        --nb[best];
        --ntot;
    }
    int ip = nfuv;
    edge[ip] = pts[0];
    for (int j = 0; j < nseg; ++j)
        for (int b = 1; b <= nb[j]; ++b)
            edge[++ip] = std::exp(std::log(pts[j]) + (std::log(pts[j + 1]) - std::log(pts[j])) * (double)b / (double)nb[j]);
    return true;
}

// photoionization_threshold_knots (ion_band_mod.f90:408-419): H, He, the
// metal thresholds in registry order, then eion_min with the FUV band.
std::vector<double> knots_of(const mochii_params& p, const std::vector<double>& metal_eth) {
    std::vector<double> knots{kEthHI, kEthHeI, kEthHeII};
    knots.insert(knots.end(), metal_eth.begin(), metal_eth.end());
    if (p.add_fuv) knots.push_back(p.eion_min);
    return knots;
}

// The luminosity sentinel and the point sources' scales (setup.f90:374-442):
// an unset par%luminosity is 1 unless an absolute (physical-type) file feeds
// the primary source; a lone point source takes the legacy scalars into slot
// 1 when src_lum(1) is unset; several sources with no src_lum split
// luminosity equally (shape spectra) or derive it from the file (absolute).
bool resolve_sources(mochii_params& q, int npt, std::string* err) {
    const bool phys = q.spectrum_type != 0;
    const bool src_abs = phys && (q.src_spectrum_file[0] || q.ion_spectrum[0]);
    if (q.luminosity < -900.0 && !(npt >= 1 && src_abs)) q.luminosity = 1.0;
    if (npt == 1) {
        if (q.src_lum[0] <= 0.0) {
            q.src_x[0] = q.xs_point;
            q.src_y[0] = q.ys_point;
            q.src_z[0] = q.zs_point;
            q.src_lum[0] = q.luminosity;
        }
    } else if (npt > 1) {
        int nset = 0;
        for (int i = 0; i < npt; ++i) nset += q.src_lum[i] > 0.0;
        if (nset == 0) {
            if (!src_abs)
                for (int i = 0; i < npt; ++i) q.src_lum[i] = q.luminosity / (double)npt;
        } else if (nset != npt) {
            return fail(err, "set par%src_lum for ALL sources or for NONE (setup.f90:428-433)");
        }
    }
    return true;
}

// source_band_luminosity (ion_band_mod.f90:379-399): an absolute spectrum
// with no scale keeps its own integral; otherwise the scale is the ionizing
// luminosity and the band carries scale / f_ion.
bool band_luminosity(const EnergyTable& t, bool is_abs, double scale, double eion_min, double* L, std::string* err) {
    if (is_abs && scale <= 0.0) {
        *L = t.total;
        return true;
    }
    const double f_ion = 1.0 - table_cdf(t, eion_min);
    if (f_ion <= 0.0) return fail(err, "cannot rescale a source with no ionizing-band luminosity (FUV-only spectrum)");
    *L = scale / f_ion;
    return true;
}

// A tabulated file slot clipped to the band (build_tabulated_band_sampler).
bool file_table(EnergyTable& t, const char* path, int icol, int ncol, const mochii_params& q, double elo,
                std::string* err) {
    std::vector<double> e, f;
    if (!spectrum_read(path, icol, ncol, q.spectrum_type, e, f, err)) return false;
    return table_band(t, e, f, elo, q.eion_max, err);
}

// build_point_source_sampler (ion_band_mod.f90:437-495): the spectrum of
// point source is (0-based) from src_spectrum_file column is + 1 >
// src_tstar(is) Planck (several components only) > ion_spectrum > tstar
// Planck, its band luminosity normalised in the branch that chose it.
bool point_sampler(const mochii_params& q, int is, bool multi, double elo, const std::vector<double>& knots,
                   EnergyTable& t, double* L, std::string* err) {
    const double scale = multi ? q.src_lum[is] : q.luminosity;
    const bool phys = q.spectrum_type != 0;
    if (q.src_spectrum_file[0]) {
        if (!file_table(t, q.src_spectrum_file, is + 1, std::max(q.nsource, 1), q, elo, err)) return false;
        return band_luminosity(t, phys, scale, q.eion_min, L, err);
    }
    if (multi && q.src_tstar[is] > 0.0) {
        if (!planck_table(t, q.src_tstar[is], elo, q.eion_max, q.source_cdf_tol, knots, err)) return false;
        return band_luminosity(t, false, scale, q.eion_min, L, err);
    }
    if (q.ion_spectrum[0]) {
        if (!file_table(t, q.ion_spectrum, 1, 1, q, elo, err)) return false;
        return band_luminosity(t, phys, scale, q.eion_min, L, err);
    }
    if (q.tstar <= 0.0) return fail(err, "point source needs a spectrum (par%tstar, par%ion_spectrum or a file)");
    if (!planck_table(t, q.tstar, elo, q.eion_max, q.source_cdf_tol, knots, err)) return false;
    return band_luminosity(t, false, scale, q.eion_min, L, err);
}

// build_external_field_sampler (ion_band_mod.f90:516-615): an ISRF preset >
// an ext_spectrum file > ext_tstar Planck > ion_spectrum > tstar Planck; the
// power entering the surface A is pi A J with an absolute J (a preset or a
// physical-type file; rescaled to ext_intensity when that is set), else
// pi J A / f_ion with J the ionizing-band intensity.
bool external_sampler(const mochii_params& q, bool sph, double elo, const std::vector<double>& knots, const double* box,
                      EnergyTable& t, double* L, std::string* err) {
    const int presid = spectrum_preset_id(q.ext_spectrum);
    const bool phys = q.spectrum_type != 0;
    const bool is_abs = presid > 0 || (phys && q.ext_spectrum[0]);
    if (presid > 0) {
        if (!preset_table(t, presid, elo, q.eion_max, q.ext_scale, err)) return false;
    } else if (q.ext_spectrum[0]) {
        if (!file_table(t, q.ext_spectrum, 1, 1, q, elo, err)) return false;
    } else if (q.ext_tstar > 0.0) {
        if (!planck_table(t, q.ext_tstar, elo, q.eion_max, q.source_cdf_tol, knots, err)) return false;
    } else if (q.ion_spectrum[0]) {
        if (!file_table(t, q.ion_spectrum, 1, 1, q, elo, err)) return false;
    } else {
        if (q.tstar <= 0.0) return fail(err, "external field needs a spectrum (par%ext_tstar / par%tstar or a file)");
        if (!planck_table(t, q.tstar, elo, q.eion_max, q.source_cdf_tol, knots, err)) return false;
    }
    if (!box) return fail(err, "external field: the box extent is unknown");
    double asurf;
    if (sph) {
        if (!(q.rmax > 0.0)) return fail(err, "ext_geometry 'sph' needs par%rmax > 0");
        if (2.0 * q.rmax > std::min(box[0], std::min(box[1], box[2])))
            return fail(err, "ext_geometry 'sph': the bounding sphere (par%rmax) must lie inside the grid");
        asurf = 4.0 * kPi * ((q.rmax * q.distance2cm) * (q.rmax * q.distance2cm));
    } else {
        const double xr = box[0] * q.distance2cm, yr = box[1] * q.distance2cm, zr = box[2] * q.distance2cm;
        asurf = 2.0 * (xr * yr + yr * zr + zr * xr);
    }
    if (is_abs) {
        *L = q.ext_intensity > 0.0 ? kPi * asurf * q.ext_intensity : kPi * asurf * t.total;
        return true;
    }
    const double f_ion = 1.0 - table_cdf(t, q.eion_min);
    if (f_ion <= 0.0) return fail(err, "the external spectrum has no luminosity inside the ionizing band");
    *L = kPi * q.ext_intensity * asurf / f_ion;
    return true;
}

// The plane-parallel slab (setup.f90:259-330, slab_setup
// ion_band_mod.f90:2083-2130, ion_setup :312-328): one component with the
// single point source's Planck spectrum at tstar, its luminosity the
// ionizing power entering one periodic tile, L = sum_face F_z A_z / f_ion,
// F_z = pi I (isotropic) or cos(theta) F_n (beam).
bool slab_build(const mochii_params& p, BandSetup& b, std::string* err, const std::vector<double>& knots,
                const double* box) {
    if (!p.xy_periodic) return fail(err, "source_geometry='slab' needs par%xy_periodic (a slab is periodic in x and y)");
    if (p.nsource > 1 || p.ext_intensity > 0.0)
        return fail(err, "source_geometry='slab' cannot be combined with point sources (nsource > 1) or an external field");
    if (p.slab_faces < 1 || p.slab_faces > 3) return fail(err, "par%slab_faces must be 'top', 'bottom' or 'both'");
    if (p.slab_nmu < 1) return fail(err, "par%slab_nmu must be >= 1");
    if (!box) return fail(err, "slab: the box extent is unknown");
    b.slab = 1;
    b.ncomp = 1;
    b.multi = 0;
    b.ext_ic = -1;
    b.qmc_ndim = 6;   // ion_qmc_ndim (:654-663): u1 energy, u2 face, u3/u4 xy, u5 mu, u6 phi
    double fz = 0.0;
    for (int f = 0; f < 2; ++f) {
        b.slab_lit[f] = (p.slab_faces >> f) & 1;
        b.slab_mode[f] = p.slab_mode[f] ? 1 : 0;
        b.slab_phi[f] = p.slab_phi[f] * (kPi / 180.0);
        b.slab_mu[f] = 1.0;
        b.slab_Fz[f] = 0.0;
        if (!b.slab_lit[f]) continue;
        if (b.slab_mode[f] == 0 && (p.slab_theta[f] < 0.0 || p.slab_theta[f] >= 90.0))
            return fail(err, "par%slab_top_theta / slab_bot_theta must lie in [0, 90) degrees for a beam");
        if (p.slab_source[f] <= 0.0) return fail(err, "par%slab_top_source / slab_bot_source must be > 0 on a lit face");
        if (b.slab_mode[f] == 1) {
            b.slab_Fz[f] = kPi * p.slab_source[f];
        } else {
            b.slab_mu[f] = std::cos(p.slab_theta[f] * (kPi / 180.0));
            b.slab_Fz[f] = b.slab_mu[f] * p.slab_source[f];
        }
        fz += b.slab_Fz[f];
    }
    b.slab_azface = (box[0] * p.distance2cm) * (box[1] * p.distance2cm);
    if (!(fz * b.slab_azface > 0.0)) return fail(err, "source_geometry='slab' has zero entering flux");
    b.slab_ptop = b.slab_Fz[0] / fz;
    const double elo = p.add_fuv ? p.efuv_min : p.eion_min;
    b.tables.assign(1, EnergyTable());
    double unused;
    mochii_params q = p;   // the spectrum resolves as point source 1's (ion_band_mod.f90:296-297)
    q.nsource = 0;
    if (!resolve_sources(q, 0, err) || !point_sampler(q, 0, false, elo, knots, b.tables[0], &unused, err))
        return false;
    const double f_ion = 1.0 - table_cdf(b.tables[0], p.eion_min);
    if (f_ion <= 0.0) return fail(err, "the slab spectrum has no luminosity inside the ionizing band");
    b.comp_x.assign(1, 0.0);
    b.comp_y.assign(1, 0.0);
    b.comp_z.assign(1, 0.0);
    b.comp_cdf.assign(1, 1.0);
    b.ion_Ltot = fz * b.slab_azface / f_ion;
    return true;
}
}  // namespace

// ion_setup + setup_continuous_source_sampler + build_point_source_sampler
// (ion_band_mod.f90:122-258, :275-353, :437-495) for internal point sources
// with Planck spectra, and ion_qmc_ndim (:654-663).
bool band_build(const mochii_params& p, BandSetup& b, std::string* err, const std::vector<double>& metal_eth,
                const double* box) {
    const int nfuv = p.add_fuv ? p.nnu_fuv : 0;
    if (p.add_fuv && p.efuv_min >= p.eion_min) return fail(err, "add_fuv requires par%efuv_min < par%eion_min");
    if (p.nnu_ion < 1) return fail(err, "par%nnu_ion must be >= 1");
    const int nnu = p.nnu_ion + nfuv;
    b.nnu_band = nnu;
    b.nfuv_band = nfuv;
    b.eedge.assign(nnu + 1, 0.0);
    const double lo = std::log(p.eion_min), hi = std::log(p.eion_max);
    for (int i = 0; i < nfuv; ++i)
        b.eedge[i] = std::exp(std::log(p.efuv_min) + (lo - std::log(p.efuv_min)) * (double)i / (double)nfuv);
    if (p.ion_align_edges) {
        if (!aligned_edges(b.eedge, nfuv, nnu, p.eion_min, p.eion_max, metal_eth, err)) return false;
    } else {
        for (int i = nfuv; i <= nnu; ++i)
            b.eedge[i] = std::exp(lo + (hi - lo) * (double)(i - nfuv) / (double)(nnu - nfuv));
    }
    if (!p.source_point && !p.source_slab)
        return fail(err, "par%source_geometry must be 'point', 'slab', 'external_rec' or 'external_sph'");
    if (p.source_slab) return slab_build(p, b, err, knots_of(p, metal_eth), box);
    // components (ion_band_mod.f90:188-199, 683-711): the point sources, then
    // the external field when it is on (external_on, :884-889)
    const bool ext_on = p.ext_intensity > 0.0 || spectrum_preset_id(p.ext_spectrum) > 0 ||
                        (p.spectrum_type != 0 && p.ext_spectrum[0]);
    if (p.source_external && !ext_on)
        return fail(err, "external source_geometry requires par%ext_intensity > 0, an ISRF preset or a physical-type "
                         "ext_spectrum (setup.f90:246-253)");
    const int npt = p.source_external ? 0 : p.nsource;
    if (npt < 0 || npt > MOCHII_MAX_SRC) return fail(err, "par%nsource out of range");
    mochii_params q = p;
    if (!resolve_sources(q, npt, err)) return false;
    b.ncomp = npt + (ext_on ? 1 : 0);
    if (b.ncomp < 1) return fail(err, "no source: par%nsource = 0 without an external field");
    b.multi = b.ncomp >= 2;
    b.ext_ic = ext_on ? b.ncomp - 1 : -1;
    b.ext_sph = p.source_external ? (p.source_external == 2) : (p.ext_geometry == 1);
    b.qmc_ndim = (b.ncomp == 1 && !ext_on) ? 3 : 7;   // ion_qmc_ndim (:654-663)
    const double elo = p.add_fuv ? p.efuv_min : p.eion_min;
    const std::vector<double> knots = knots_of(p, metal_eth);
    b.tables.assign(b.ncomp, EnergyTable());
    b.comp_x.assign(b.ncomp, 0.0);
    b.comp_y.assign(b.ncomp, 0.0);
    b.comp_z.assign(b.ncomp, 0.0);
    std::vector<double> L(b.ncomp);
    for (int c = 0; c < b.ncomp; ++c) {
        if (c == b.ext_ic) {
            if (!external_sampler(q, b.ext_sph, elo, knots, box, b.tables[c], &L[c], err)) return false;
            continue;
        }
        if (!point_sampler(q, c, b.multi, elo, knots, b.tables[c], &L[c], err)) return false;
        b.comp_x[c] = b.multi ? q.src_x[c] : q.xs_point;
        b.comp_y[c] = b.multi ? q.src_y[c] : q.ys_point;
        b.comp_z[c] = b.multi ? q.src_z[c] : q.zs_point;
    }
    b.ion_Ltot = 0.0;
    for (double x : L) b.ion_Ltot += x;
    b.comp_cdf.assign(b.ncomp, 1.0);
    if (b.multi) {
        b.comp_cdf[0] = L[0];
        for (int c = 1; c < b.ncomp; ++c) b.comp_cdf[c] = b.comp_cdf[c - 1] + L[c];
        const double last = b.comp_cdf[b.ncomp - 1];
        for (auto& x : b.comp_cdf) x = x / last;
    }
    return true;
}

}  // namespace mochii
