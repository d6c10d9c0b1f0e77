// The rates file of a finished run (gas_rates_write, gas_rates_mod.f90:
// 216-366, with species_write, species_mod.f90:873-916): the same datasets
// and header keywords as the reference's FITS/HDF5 image file, written
// without an I/O library as a directory <base>_rates/ holding one NumPy
// .npy file per dataset (little-endian FP64, C order) and header.json (the
// run's keywords, and per dataset its file, shape, comment and keywords).
//
// Shapes follow the reference's arrays in their memory order: a Fortran
// array a(n1, n2) is stored as shape (n2, n1), so that element (i, j) of the
// reference is [j-1][i-1] here and the bytes are the reference's bytes --
// J_nu(nnu_band, nleaf) -> (nleaf, nnu_band), LeafXYZ(nleaf, 3) -> (3, nleaf),
// x_<el>_stages(nstage, nleaf) -> (nleaf, nstage).
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "ctx.h"
#include "mochii_gpu.h"
#include "transport.h"
#include "physics.cuh"

namespace mochii {
namespace {

// One dataset: its extension name, comment, shape and values.
struct Dataset {
    std::string name, comment;
    std::vector<long long> shape;
    std::vector<double> v;
    std::string keywords;   // extra JSON members ("ABUND": ...), or empty
};

std::string json_str(const std::string& s) {
    std::string o = "\"";
    for (char ch : s) {
        if (ch == '"' || ch == '\\') o += '\\';
        o += ch;
    }
    return o + "\"";
}

std::string json_num(double x) {
    if (!std::isfinite(x)) return "null";
    char b[40];
    std::snprintf(b, sizeof(b), "%.17g", x);
    return b;
}

// NumPy format 1.0: magic, header length, the header dict padded so the
// data starts on a 64-byte boundary, then the raw values.
bool write_npy(const std::string& path, const Dataset& d) {
    std::string shape = "(";
    for (size_t i = 0; i < d.shape.size(); ++i) shape += std::to_string(d.shape[i]) + (d.shape.size() == 1 ? "," : i + 1 < d.shape.size() ? ", " : "");
    shape += ")";
    std::string hdr = "{'descr': '<f8', 'fortran_order': False, 'shape': " + shape + ", }";
    const size_t pre = 10;
    size_t total = pre + hdr.size() + 1;
    const size_t pad = (64 - total % 64) % 64;
    hdr += std::string(pad, ' ') + "\n";
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
    const unsigned short hl = (unsigned short)hdr.size();
    bool ok = std::fwrite(magic, 1, 8, f) == 8;
    ok = ok && std::fwrite(&hl, 2, 1, f) == 1;
    ok = ok && std::fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size();
    ok = ok && std::fwrite(d.v.data(), 8, d.v.size(), f) == d.v.size();
    return std::fclose(f) == 0 && ok;
}

const char* element_name(int Z) {   // the registry's names (element_<el>.txt, ELEMENT line)
    switch (Z) {
        case 6: return "c";
        case 7: return "n";
        case 8: return "o";
        case 10: return "ne";
        case 12: return "mg";
        case 14: return "si";
        case 16: return "s";
        case 17: return "cl";
        case 18: return "ar";
        case 20: return "ca";
        case 26: return "fe";
        default: return "x";
    }
}

}  // namespace
}  // namespace mochii

using namespace mochii;

extern "C" int mochii_write_rates(mochii_ctx* c, const char* base, const mochii_run_info* run) {
    if (!c || !base || !base[0]) return MOCHII_ERR_BAD_PARAM;
    const long long nl = c->grid.nleaf;
    const int nnu = c->nnu;
    std::vector<Dataset> ds;
    auto field = [&](const char* fname, const char* ext, const char* comment) -> int {
        Dataset d{ext, comment, {nl}, std::vector<double>((size_t)nl), ""};
        const int rc = mochii_get_field(c, fname, d.v.data(), nl);
        if (rc == MOCHII_OK) ds.push_back(std::move(d));
        return rc;
    };
    int rc = MOCHII_OK;
    const char* rate_fields[6][3] = {
        {"gamma_HI", "Gamma_HI", "H I photoionization rate [s^-1]"},
        {"gamma_HeI", "Gamma_HeI", "He I photoionization rate [s^-1]"},
        {"gamma_HeII", "Gamma_HeII", "He II photoionization rate [s^-1]"},
        {"heat_HI", "Heat_HI", "H I photoheating [erg/s per HI]"},
        {"heat_HeI", "Heat_HeI", "He I photoheating [erg/s per HeI]"},
        {"heat_HeII", "Heat_HeII", "He II photoheating [erg/s per HeII]"}};
    for (auto& f : rate_fields)
        if ((rc = field(f[0], f[1], f[2]))) return rc;
    if (c->par.ion_add_dust && (rc = field("heat_dust", "Heat_dust", "grain heating [erg/s/cm^3]"))) return rc;
    // dust_temp_compute at output (main.f90:241-248), then its dataset (gas_rates_mod.f90:287-293)
    if (c->par.ion_add_dust && (rc = field("T_dust", "T_dust", "equilibrium mixture dust temperature [K]"))) return rc;

    // geometry: leaf centres and half widths
    std::vector<double> half((size_t)nl), cx((size_t)nl), cy((size_t)nl), cz((size_t)nl);
    if ((rc = mochii_get_field(c, "leaf_half", half.data(), nl))) return rc;
    if (c->oct.ncells > 0) {
        std::vector<double4> g((size_t)nl);
        if (cudaMemcpy(g.data(), c->oct.lgeo, (size_t)nl * sizeof(double4), cudaMemcpyDeviceToHost) != cudaSuccess)
            return MOCHII_ERR_CUDA;
        for (long long i = 0; i < nl; ++i) {
            cx[i] = g[i].x;
            cy[i] = g[i].y;
            cz[i] = g[i].z;
        }
    } else {
        const Grid& G = c->grid;
        for (long long il = 0; il < nl; ++il) {
            const long long ix = il % G.nx, iy = (il / G.nx) % G.ny, iz = il / ((long long)G.nx * G.ny);
            cx[il] = G.xmin + (ix + 0.5) * G.dcell;
            cy[il] = G.ymin + (iy + 0.5) * G.dcell;
            cz[il] = G.zmin + (iz + 0.5) * G.dcell;
        }
    }

    // J_nu(nnu_band, nleaf) = jt_ion / (4 pi (2 h)^3 dnu d2cm^2)  (gas_rates_mod.f90:296-305)
    const std::vector<double>& edge = c->band.eedge;
    std::vector<double> ebin((size_t)nnu), dbin((size_t)nnu), dnu((size_t)nnu);
    for (int i = 0; i < nnu; ++i) {   // ion_band_mod.f90:181-186
        ebin[i] = std::sqrt(edge[i] * edge[i + 1]);
        dbin[i] = edge[i + 1] - edge[i];
        dnu[i] = dbin[i] * kEv2erg / kHPlanck;
    }
    {
        Dataset d{"J_nu", "J(nu,leaf) [erg/s/cm^2/Hz/sr]", {nl, nnu}, std::vector<double>((size_t)nl * nnu), ""};
        if ((rc = mochii_get_field(c, "jt_ion", d.v.data(), (int64_t)nl * nnu))) return rc;
        const double d2 = c->par.distance2cm * c->par.distance2cm;
        const double fourpi = 4.0 * kPi;
        for (long long il = 0; il < nl; ++il) {
            const double w = 2.0 * half[il];
            for (int i = 0; i < nnu; ++i) d.v[(size_t)il * nnu + i] /= fourpi * (w * w * w) * dnu[i] * d2;
        }
        ds.push_back(std::move(d));
    }
    const char* state_fields[5][3] = {{"x_HI", "x_HI", "n_HI/n_H per leaf"},
                                      {"x_HeI", "x_HeI", "n_HeI/n_He per leaf"},
                                      {"x_HeII", "x_HeII", "n_HeII/n_He per leaf"},
                                      {"n_e", "n_e", "electron density [cm^-3]"},
                                      {"T_e", "T_e", "electron temperature [K]"}};
    for (auto& f : state_fields)
        if ((rc = field(f[0], f[1], f[2]))) return rc;
    ds.push_back(Dataset{"E_bin", "bin centers [eV]", {nnu}, ebin, ""});
    ds.push_back(Dataset{"dE_bin", "bin widths [eV]", {nnu}, dbin, ""});
    {
        Dataset d{"LeafXYZ", "leaf center x,y,z (code units)", {3, nl}, std::vector<double>((size_t)3 * nl), ""};
        std::memcpy(d.v.data(), cx.data(), nl * 8);
        std::memcpy(d.v.data() + nl, cy.data(), nl * 8);
        std::memcpy(d.v.data() + 2 * nl, cz.data(), nl * 8);
        ds.push_back(std::move(d));
        Dataset s{"LeafSize", "leaf full width (code units)", {nl}, std::vector<double>((size_t)nl), ""};
        for (long long i = 0; i < nl; ++i) s.v[i] = 2.0 * half[i];
        ds.push_back(std::move(s));
    }
    // species_write: per element the stage fractions of the written state,
    // its photoionization and photoheating rates
    if (c->metal.ntr > 0) {
        const int ntr = c->metal.ntr, nst = c->metal.nst;
        std::vector<double> xm((size_t)nl * nst), gm((size_t)nl * ntr), hm((size_t)nl * ntr);
        if ((rc = mochii_get_field(c, "x_metal", xm.data(), (int64_t)nl * nst))) return rc;
        if ((rc = mochii_get_field(c, "gamma_metal", gm.data(), (int64_t)nl * ntr))) return rc;
        if ((rc = mochii_get_field(c, "heat_metal", hm.data(), (int64_t)nl * ntr))) return rc;
        int s0 = 0, t0 = 0;
        for (const MetalEl& e : c->species.el) {
            const std::string nm = element_name(e.Z);
            const int ns = e.nstage, nt = e.nstage - 1;
            Dataset x{"x_" + nm + "_stages", "ion fractions (stage, leaf)", {nl, ns}, std::vector<double>((size_t)nl * ns),
                      "\"ABUND\": " + json_num(e.abund)};
            Dataset g{"Gamma_" + nm + "_stages", "photoionization rates (transition, leaf) [s^-1]", {nl, nt},
                      std::vector<double>((size_t)nl * nt), ""};
            Dataset h{"Heat_" + nm + "_stages", "photoheating rates (transition, leaf) [erg/s per ion]", {nl, nt},
                      std::vector<double>((size_t)nl * nt), ""};
            for (long long il = 0; il < nl; ++il) {
                for (int i = 0; i < ns; ++i) x.v[(size_t)il * ns + i] = xm[(size_t)il * nst + s0 + i];
                for (int i = 0; i < nt; ++i) {
                    g.v[(size_t)il * nt + i] = gm[(size_t)il * ntr + t0 + i];
                    h.v[(size_t)il * nt + i] = hm[(size_t)il * ntr + t0 + i];
                }
            }
            ds.push_back(std::move(x));
            ds.push_back(std::move(g));
            ds.push_back(std::move(h));
            s0 += ns;
            t0 += nt;
        }
    }

    // the directory, the datasets, the header
    const std::string dir = std::string(base) + "_rates";
    if (::mkdir(dir.c_str(), 0755) != 0 && errno != EEXIST) {
        c->last_error = "mochii_write_rates: cannot create " + dir;
        return MOCHII_ERR_BAD_PARAM;
    }
    for (const Dataset& d : ds) {
        if (!write_npy(dir + "/" + d.name + ".npy", d)) {
            c->last_error = "mochii_write_rates: cannot write " + dir + "/" + d.name + ".npy";
            return MOCHII_ERR_BAD_PARAM;
        }
    }
    const mochii_pass_stats& ps = c->last_pass;
    const mochii_params& p = c->par;
    mochii_run_info ri = {};
    if (run) ri = *run;
    std::string j = "{\n  \"format\": \"mochii rates: one .npy per dataset (FP64, C order; a Fortran a(n1,n2) is "
                    "shape (n2,n1)), keywords of the reference's rates file\",\n  \"keywords\": {\n";
    auto kv = [&](const std::string& k, const std::string& v, const std::string& comment, bool last = false) {
        j += "    " + json_str(k) + ": {\"value\": " + v + ", \"comment\": " + json_str(comment) + "}" +
             (last ? "\n" : ",\n");
    };
    kv("NNU_ION", std::to_string(p.nnu_ion), "ionizing energy-bin count");
    kv("NNU_BAND", std::to_string(nnu), "total band bins (ionizing+FUV)");
    kv("EION_MIN", json_num(p.eion_min), "band lower edge [eV]");
    kv("EION_MAX", json_num(p.eion_max), "band upper edge [eV]");
    kv("TOT_LUM", json_num(p.luminosity), "band luminosity [erg/s]");
    kv("DIST_CM", json_num(p.distance2cm), "distance unit (cm)");
    kv("nphotons", std::to_string((long long)p.nphotons), "number of photons");
    kv("CONVERGD", ri.converged ? "true" : "false", "gas iteration converged");
    kv("NITERDON", std::to_string(ri.iterations), "gas iterations run");
    kv("FINALDX", json_num(ri.final_dx), "final max|delta x_HII|");
    kv("FINALDTE", json_num(ri.final_dte), "final max|delta Te|/Te");
    kv("FLDCONS", ri.field_consistent ? "true" : "false", "rates rebuilt by transporting the written state");
    kv("IONEMODE", json_str("continuous"), "ionizing packet energy sampling");
    kv("CDFRTOL", json_num(p.source_cdf_tol), "source sampler relative tolerance");
    kv("NUBINUSE", json_str("diagnostic_only"), "role of ionizing spectral bins");
    kv("ENRGSAMP", json_str(p.launch_sobol ? "sobol" : "random"), "energy/source sampling sequence");
    kv("L_EMIT", json_num(ps.energy_emitted), "transported ionizing packet luminosity");
    kv("L_ABS", json_num(ps.energy_absorbed), "absorbed ionizing packet luminosity");
    kv("L_ESC", json_num(ps.energy_escaped), "escaped ionizing packet luminosity", !p.launch_sobol);
    if (p.launch_sobol) kv("QMCSEED", std::to_string(p.qmc_seed), "Sobol scramble seed", true);
    j += "  },\n  \"datasets\": [\n";
    for (size_t i = 0; i < ds.size(); ++i) {
        const Dataset& d = ds[i];
        std::string shape = "[";
        for (size_t k = 0; k < d.shape.size(); ++k) shape += std::to_string(d.shape[k]) + (k + 1 < d.shape.size() ? ", " : "");
        shape += "]";
        j += "    {\"EXTNAME\": " + json_str(d.name) + ", \"file\": " + json_str(d.name + ".npy") + ", \"shape\": " + shape +
             ", \"comment\": " + json_str(d.comment) + (d.keywords.empty() ? "" : ", " + d.keywords) + "}" +
             (i + 1 < ds.size() ? ",\n" : "\n");
    }
    j += "  ]\n}\n";
    FILE* f = std::fopen((dir + "/header.json").c_str(), "w");
    if (!f || std::fwrite(j.data(), 1, j.size(), f) != j.size() || std::fclose(f) != 0) {
        c->last_error = "mochii_write_rates: cannot write " + dir + "/header.json";
        return MOCHII_ERR_BAD_PARAM;
    }
    return MOCHII_OK;
}

// The grains' infrared spectrum of the current T_dust (dust_ir_write,
// dust_temp_mod.f90:173-214): lam[240] [um], lnu[240] [erg/s/Hz] and
// labs_lir[2] = the absorbed power sum Heat_dust V and the trapezoid integral
// of L_nu over frequency [erg/s].
extern "C" int mochii_dust_ir(mochii_ctx* c, double* lam, double* lnu, double* labs_lir) {
    if (!c || !lam || !lnu || !labs_lir) return MOCHII_ERR_BAD_PARAM;
    if (!c->par.ion_add_dust || !c->rhokap) {
        c->last_error = "mochii_dust_ir: needs par%ion_add_dust";
        return MOCHII_ERR_BAD_PARAM;
    }
    double* d = nullptr;
    std::vector<double> out(kDustIrN + 1);
    cudaError_t e = dust_temp_launch(c);
    if (e == cudaSuccess) e = cudaMallocAsync(&d, (kDustIrN + 1) * 8, c->stream);
    if (e == cudaSuccess) e = dust_ir_launch(c, d);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), d, (kDustIrN + 1) * 8, cudaMemcpyDeviceToHost, c->stream);
    if (d) cudaFreeAsync(d, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        c->last_error = std::string("mochii_dust_ir: ") + cudaGetErrorString(e);
        return MOCHII_ERR_CUDA;
    }
    double lir = 0.0;
    for (int k = 0; k < kDustIrN; ++k) {
        lam[k] = c->tdust_host.lam_ir[k];
        lnu[k] = out[k];
    }
    for (int k = 0; k + 1 < kDustIrN; ++k) {
        const double dnu = 2.99792458e10 / (lam[k] * 1.0e-4) - 2.99792458e10 / (lam[k + 1] * 1.0e-4);
        lir = lir + 0.5 * (lnu[k] + lnu[k + 1]) * dnu;
    }
    labs_lir[0] = out[kDustIrN];
    labs_lir[1] = lir;
    return MOCHII_OK;
}

// dust_ir_write's text file <base>_dustir.txt: two header lines with the
// absorbed power, the integral of L_nu and their ratio, then lambda [um] and
// L_nu [erg/s/Hz] per line.
extern "C" int mochii_write_dust_ir(mochii_ctx* c, const char* base) {
    if (!c || !base || !base[0]) return MOCHII_ERR_BAD_PARAM;
    double lam[kDustIrN], lnu[kDustIrN], ab[2];
    const int rc = mochii_dust_ir(c, lam, lnu, ab);
    if (rc) return rc;
    const std::string path = std::string(base) + "_dustir.txt";
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) {
        c->last_error = "cannot write " + path;
        return MOCHII_ERR_BAD_PARAM;
    }
    std::fprintf(f, "# MoCHII equilibrium-mixture dust IR spectrum (single T_d per leaf; SEDust stochastic/PAH "
                    "bands are the next stage)\n");
    std::fprintf(f, "# L_abs(dust) = %14.6E erg/s;  integral L_nu dnu = %14.6E;  ratio = %7.3f\n", ab[0], ab[1],
                 ab[1] / std::max(ab[0], 2.2250738585072014e-308));
    std::fprintf(f, "# lambda[um]   L_nu[erg/s/Hz]\n");
    for (int k = 0; k < kDustIrN; ++k) std::fprintf(f, "%12.4f%15.6E\n", lam[k], lnu[k]);
    return std::fclose(f) == 0 ? MOCHII_OK : MOCHII_ERR_BAD_PARAM;
}

extern "C" int mochii_slab_tally(mochii_ctx* c, double* iesc, int n, double* meta) {
    if (!c) return MOCHII_ERR_BAD_PARAM;
    if (!c->band.slab || !c->slab_iesc) {
        c->last_error = "the boundary tally needs par%source_geometry = 'slab'";
        return MOCHII_ERR_BAD_PARAM;
    }
    if (n != (int)c->slab_host.size() || (!iesc && n > 0)) {
        c->last_error = "mochii_slab_tally: n must be 2 * par%slab_nmu";
        return MOCHII_ERR_BAD_PARAM;
    }
    for (int k = 0; k < n; ++k) iesc[k] = c->slab_host[k];
    if (meta) {
        meta[0] = c->band.ion_Ltot;
        meta[1] = c->band.slab_azface;
    }
    return MOCHII_OK;
}

extern "C" int mochii_write_slab_imu(mochii_ctx* c, const char* base) {
    if (!c || !base || !base[0]) return MOCHII_ERR_BAD_PARAM;
    const int n = (int)c->slab_host.size();
    std::vector<double> v(std::max(n, 1));
    double meta[2];
    const int rc = mochii_slab_tally(c, v.data(), n, meta);
    if (rc) return rc;
    const int nmu = n / 2;
    const double lin = meta[0], az = meta[1], dmu = 1.0 / (double)nmu;
    double top = 0.0, bot = 0.0;
    for (int k = 0; k < nmu; ++k) {
        top += v[k];
        bot += v[nmu + k];
    }
    const double labs = lin - top - bot;
    const bool lit_top = c->band.slab_lit[0], lit_bot = c->band.slab_lit[1];
    const std::string path = std::string(base) + "_slab_Imu.txt";
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) {
        c->last_error = "cannot write " + path;
        return MOCHII_ERR_BAD_PARAM;
    }
    std::fprintf(f, "# MoCHII plane-parallel slab: emergent intensity I(mu) at the z-boundaries.\n");
    std::fprintf(f, "# L_in           [erg/s] = %14.6E\n", lin);
    std::fprintf(f, "# L_escape_top   [erg/s] = %14.6E   fraction = %8.5f\n", top, top / lin);
    std::fprintf(f, "# L_escape_bottom[erg/s] = %14.6E   fraction = %8.5f\n", bot, bot / lin);
    std::fprintf(f, "# L_absorbed     [erg/s] = %14.6E   fraction = %8.5f\n", labs, labs / lin);
    if (lit_top != lit_bot) {   // one lit face: escape there is reflected, at the other transmitted
        const double refl = lit_top ? top : bot, tran = lit_top ? bot : top;
        std::fprintf(f, lit_top ? "# illuminated face = top: escape at top = reflected, at bottom = transmitted.\n"
                                : "# illuminated face = bottom: escape at bottom = reflected, at top = transmitted.\n");
        std::fprintf(f, "# L_reflected    [erg/s] = %14.6E   fraction = %8.5f\n", refl, refl / lin);
        std::fprintf(f, "# L_transmitted  [erg/s] = %14.6E   fraction = %8.5f\n", tran, tran / lin);
    } else {
        std::fprintf(f, "# both (or neither) faces illuminated: the top and bottom escape each mix\n");
        std::fprintf(f, "# reflection and transmission and are not separable without an incident-face tag.\n");
    }
    std::fprintf(f, "# A_zface        [cm^2]  = %14.6E\n", az);
    std::fprintf(f, "#   mu        I_top[erg/s/cm^2/sr]   I_bot[erg/s/cm^2/sr]\n");
    for (int k = 0; k < nmu; ++k) {
        const double mu = ((double)(k + 1) - 0.5) * dmu;
        const double norm = az * kTwoPi * mu * dmu;
        std::fprintf(f, "%8.5f%22.8E%22.8E\n", mu, v[k] / norm, v[nmu + k] / norm);
    }
    return std::fclose(f) == 0 ? MOCHII_OK : MOCHII_ERR_BAD_PARAM;
}
