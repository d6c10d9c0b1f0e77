// C-ABI layer: context life cycle, the replaced module entry points and the
// state-exchange / test hooks declared in include/mochii_gpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "band.h"
#include "ctx.h"
#include "mochii_gpu.h"
#include "physics.cuh"
#include "qmc.cuh"
#include "species.h"
#include "thermal.h"
#include "transport.h"

using namespace mochii;

namespace {

thread_local std::string g_init_error;

int fail(mochii_ctx* c, int code, const std::string& msg) {
    if (c) c->last_error = msg; else g_init_error = msg;
    return code;
}

#define CK(c, call)                                                                              \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail((c), MOCHII_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
cudaError_t dalloc(T** p, size_t n) {
    return cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T) + 16);
}

// Bytes of the metal moment tallies: nmb bins per leaf of kMomDeg FP64 words
// (or compensated FP32 pairs), or with FP32 moments 8 floats (6 used) so a
// bin's update is one aligned 32-byte sector.
size_t mom_bytes(const mochii_ctx* c) {
    const MetalDev& m = c->metal;
    return (size_t)c->grid.nleaf * m.nmb * (m.mom32 ? 8 * sizeof(float) : kMomDeg * 8);
}

// Bytes of the exact metal tallies: two words (Gamma, heating path sums) per
// transition slot, FP64 (or a compensated FP32 pair), or FP32 with raw32.
size_t raw_bytes(const mochii_ctx* c) {
    const MetalDev& m = c->metal;
    return (size_t)c->grid.nleaf * m.ntrp * 2 * (m.raw32 ? sizeof(float) : 8);
}

void free_records(mochii_ctx* c) {
    for (void* q : {(void*)c->rec.tm, (void*)c->rec.td, (void*)c->rec.cell, (void*)c->rec.bits, c->rec.sig, c->rec.coef,
                    (void*)c->rec.E, c->rec.msig, c->rec.dsc, (void*)c->rec.p0, (void*)c->rec.key,
                    (void*)c->rec.key_sorted, (void*)c->rec.seq, (void*)c->rec.perm, c->rec.sort_tmp})
        if (q) cudaFree(q);
    c->rec = RecordBuffers();
}

// Launch records of one chunk of up to cap packets (transport.cu).
cudaError_t alloc_records(mochii_ctx* c, long long cap) {
    const size_t rsz = c->fp32 ? 4 : 8;
    c->rec.cap = cap;
    cudaError_t e;
    if ((e = dalloc(&c->rec.tm, 3 * (size_t)cap)) != cudaSuccess) return e;
    if ((e = dalloc(&c->rec.td, 3 * (size_t)cap)) != cudaSuccess) return e;
    if ((e = dalloc(&c->rec.cell, (size_t)cap)) != cudaSuccess) return e;
    if ((e = dalloc(&c->rec.bits, (size_t)cap)) != cudaSuccess) return e;
    const size_t nsig = c->xscore ? 4 : 3, ncoef = c->xscore ? 8 : 6;   // + grain / FUV rows
    if ((e = cudaMalloc(&c->rec.sig, nsig * (size_t)cap * rsz + 64)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&c->rec.coef, ncoef * (size_t)cap * rsz + 64)) != cudaSuccess) return e;
    if (c->scatter && (e = cudaMalloc(&c->rec.dsc, 2 * (size_t)cap * rsz + 64)) != cudaSuccess) return e;
    if ((c->scatter || c->par.ion_peel || c->band.slab) && c->oct.ncells == 0 &&
        (e = dalloc(&c->rec.p0, 6 * (size_t)cap)) != cudaSuccess)
        return e;
    if (c->metal.ntr > 0) {
        if ((e = dalloc(&c->rec.E, (size_t)cap)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&c->rec.msig, (size_t)c->metal.ntrp * cap * rsz + 64)) != cudaSuccess) return e;
    }
    if (c->par.packet_order && (e = packet_order_alloc(c, cap)) != cudaSuccess) return e;
    return cudaSuccess;
}

void release(mochii_ctx* c) {
    if (!c) return;
    void* ptrs[] = {c->nH, c->xHI, c->xHeI, c->xHeII, c->ne, c->Te, c->col, c->tally, c->jt, c->rates,
                    c->tab.tab_e, c->tab.tab_f, c->tab.tab_c, c->tab.tab_off, c->tab.comp, c->tab.eedge,
                    c->tab.qmc, c->tw.ledger, c->tw.counters, c->bw.partial, c->bw.counters,
                    c->bw.work, c->bw.work_sorted, c->bw.iota, c->bw.order, c->bw.sort_tmp, c->bw.next,
                    c->rec.tm, c->rec.td, c->rec.cell, c->rec.bits, c->rec.sig, c->rec.coef,
                    c->th.gff, c->th.lamref, c->th.Ssup, c->th.tinv,
                    c->dif.ch, c->dif.tot, c->dif.scan_tmp, c->dif.tables, c->dif.he_tab,
                    (void*)c->metal.el, c->metal.egam, c->metal.eheat, c->metal.opac, c->metal.raw,
                    (void*)c->metal.medge, c->metal.mom, c->twarm, c->twarm_err, c->tdust, c->tdust_tab,
                    (void*)c->rec.E, c->rec.msig, c->oct_blob, c->rec.dsc, (void*)c->rec.p0,
                    (void*)c->dust_blob, (void*)c->rhokap, (void*)c->ttab, (void*)c->metal_lnl,
                    (void*)c->th.lnL, (void*)c->rec.key, (void*)c->rec.key_sorted, (void*)c->rec.seq,
                    (void*)c->rec.perm, c->rec.sort_tmp, c->peel_blob, (void*)c->slab_iesc};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (cudaEvent_t e : {c->ev0, c->ev1, c->evA, c->evB})
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
}

// Checks read_input applies (setup.f90:76-626) plus the extent of this build.
int validate(const mochii_params& p, std::string* why, int* code) {
    *code = MOCHII_ERR_BAD_PARAM;
    if (p.nphotons < 1) return *why = "par%no_photons must be >= 1", 1;
    if (p.eion_max <= p.eion_min || p.eion_min <= 0.0) return *why = "need 0 < par%eion_min < par%eion_max", 1;
    if (p.grid_car) {
        if (p.xmax <= 0.0 || p.nx < 1 || p.ny < 1 || p.nz < 1) return *why = "car grid needs par%xmax > 0 and nx,ny,nz >= 1", 1;
        if (p.nx > 1024 || p.ny > 1024 || p.nz > 1024) return *why = "car grid: nx, ny, nz must be <= 1024", 1;
        const double dcx = 2.0 * p.xmax / p.nx, dcy = 2.0 * p.ymax / p.ny, dcz = 2.0 * p.zmax / p.nz;
        if (std::fabs(dcy - dcx) > 1.0e-9 * dcx || std::fabs(dcz - dcx) > 1.0e-9 * dcx)
            return *why = "car grid needs cubic cells: 2*xmax/nx = 2*ymax/ny = 2*zmax/nz", 1;   // grid_mod_amr.f90:91-96
    }
    if (p.ion_relax <= 0.0 || p.ion_relax > 1.0) return *why = "par%ion_relax must lie in (0, 1]", 1;
    if (p.te_fixed <= 0.0) return *why = "par%te_fixed must be positive", 1;
    if (p.solve_te && !(p.te_min > 0.0 && p.te_max > p.te_min)) return *why = "need 0 < par%te_min < par%te_max", 1;
    if (p.He_abund < 0.0) return *why = "par%He_abund must be >= 0", 1;
    if (!p.grid_car && !p.amr_file[0]) return *why = "grid_type='amr' needs par%amr_file (a text leaf list)", 1;
    if (spectrum_preset_id(p.ion_spectrum) > 0 || spectrum_preset_id(p.src_spectrum_file) > 0)   // setup.f90:224-232
        return *why = "ISRF preset names (draine/habing/mathis) are valid only for par%ext_spectrum", 1;
    if (spectrum_preset_id(p.ext_spectrum) > 0) {   // setup.f90:339-352
        if (p.ext_scale <= 0.0) return *why = "par%ext_scale must be > 0 for an ISRF preset", 1;
        if (!p.add_fuv)
            return *why = "the ISRF presets are FUV-only; set par%add_fuv (with par%efuv_min < 13.6)", 1;
    }
    if (p.source_slab) {   // setup.f90:259-327
        if (!p.xy_periodic) return *why = "source_geometry='slab' needs par%xy_periodic (a slab is periodic in x and y)", 1;
        if (p.nsource > 1 || p.ext_intensity > 0.0)
            return *why = "source_geometry='slab' cannot be combined with point sources (nsource > 1) or an external field", 1;
        if (p.slab_nmu < 1) return *why = "par%slab_nmu must be >= 1", 1;
        for (int f = 0; f < 2; ++f) {
            if (!((p.slab_faces >> f) & 1)) continue;
            if (!p.slab_mode[f] && (p.slab_theta[f] < 0.0 || p.slab_theta[f] >= 90.0))
                return *why = "par%slab_top_theta / slab_bot_theta must lie in [0, 90) degrees for a beam", 1;
            if (p.slab_source[f] <= 0.0) return *why = "par%slab_top_source / slab_bot_source must be > 0 on a lit face", 1;
        }
    }
    *code = MOCHII_ERR_UNSUPPORTED;
    if (!p.source_point && !p.source_slab) return *why = "only point sources, external fields and the slab are built", 1;
    if (!p.launch_sobol) return *why = "launch_sequence='random' is not built; use 'sobol'", 1;
    if (p.ion_add_dust && p.dust_law == 2)
        return *why = "dust_density_law: only 'global_dgr' and 'none' are built", 1;
    if (p.ion_add_dust && (p.taumax > 0.0 || p.tauhomo > 0.0))
        return *why = "the taumax / tauhomo dust normalisations are not built", 1;
    if (p.ion_add_dust && !p.ion_dust_kext[0])
        return *why = "ion_add_dust needs par%ion_dust_kext (the grain-model optics are not built)", 1;
    *code = MOCHII_ERR_BAD_PARAM;
    if (p.ion_peel && p.xy_periodic)   // setup.f90:531-539
        return *why = "par%ion_peel is not supported with par%xy_periodic (use the slab's boundary I(mu) tally)", 1;
    *code = MOCHII_ERR_UNSUPPORTED;
    if (p.use_sec_ion) return *why = "use_sec_ion is not built in this library version", 1;
    if (p.grain_pe) return *why = "grain_pe is not built in this library version", 1;
    return 0;
}

}  // namespace

extern "C" const char* mochii_strerror(int s) {
    switch (s) {
        case MOCHII_OK: return "ok";
        case MOCHII_ERR_BAD_PARAM: return "bad parameter";
        case MOCHII_ERR_TABLE: return "data table error";
        case MOCHII_ERR_CUDA: return "CUDA runtime error";
        case MOCHII_ERR_TIMEOUT: return "device loop hit its iteration cap";
        case MOCHII_ERR_NONFINITE: return "non-finite value";
        case MOCHII_ERR_CLOSURE: return "energy closure exceeds 5e-13";
        case MOCHII_ERR_NOT_CONVERGED: return "iteration did not converge";
        case MOCHII_ERR_UNSUPPORTED: return "configuration outside the built path";
        case MOCHII_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

extern "C" const char* mochii_last_error(const mochii_ctx* c) {
    return c ? c->last_error.c_str() : g_init_error.c_str();
}

extern "C" int mochii_init(const mochii_params* pin, mochii_ctx** out) {
    if (!pin || !out) return fail(nullptr, MOCHII_ERR_BAD_PARAM, "null argument");
    *out = nullptr;
    std::string why;
    int code;
    if (validate(*pin, &why, &code)) return fail(nullptr, code, why);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return fail(nullptr, MOCHII_ERR_NO_DEVICE, "no CUDA device is visible");
    }
    auto* c = new mochii_ctx();
    c->par = *pin;
    mochii_params& p = c->par;
    if (p.diffuse_field) p.caseA = 1;   // setup.f90:580-583: the diffuse field forces case A
    // species before the band (main.f90:64-83): the metal thresholds pin
    // band edges and sampler knots
    if (p.use_metals && !species_build(p, c->species, &why)) {
        delete c;
        return fail(nullptr, MOCHII_ERR_TABLE, why);
    }
    cudaGetDevice(&c->device);
    Grid& g = c->grid;
    // octree from a text leaf list (grid_mod_amr.f90:50-62, read_generic_amr.f90:60-81,
    // octree_mod.f90:342-479): leaf centres, levels and n_H from the file
    std::vector<double> lx, ly, lz, lnH;
    OctHost oh;
    if (!p.grid_car) {
        std::vector<int> lev;
        double boxlen = 0.0;
        bool read_ok;
        if (g_leaf_preload) {   // the refined leaves of mochii_refine_front
            lx = *g_leaf_preload->x; ly = *g_leaf_preload->y; lz = *g_leaf_preload->z;
            lev = *g_leaf_preload->lev; lnH = *g_leaf_preload->nH;
            boxlen = g_leaf_preload->boxlen;
            read_ok = true;
        } else {
            read_ok = leaf_list_read(p.amr_file, lx, ly, lz, lev, lnH, &boxlen, &why);
        }
        if (!read_ok || !octree_build(lx, ly, lz, lev, 0.5 * boxlen, oh, &why)) {
            delete c;
            return fail(nullptr, MOCHII_ERR_BAD_PARAM, why);
        }
        const double half = 0.5 * boxlen;
        p.xmax = p.ymax = p.zmax = half;
        g.nx = g.ny = g.nz = 0;
        g.nleaf = oh.nleaf;
        g.xmin = g.ymin = g.zmin = -half;
        g.xmax = g.ymax = g.zmax = half;
        g.dcell = 0.0;
        c->lhalf.resize(oh.nleaf);
        for (int l = 0; l < oh.nleaf; ++l) c->lhalf[l] = oh.lgeo[4 * (size_t)l + 3];
    } else {
        // namelist car grid, grid_mod_amr.f90:64-133 and amr_build_car (octree_mod.f90:648-674)
        g.nx = p.nx; g.ny = p.ny; g.nz = p.nz;
        g.nleaf = (long long)p.nx * p.ny * p.nz;
        g.xmin = -p.xmax; g.xmax = p.xmax;
        g.ymin = -p.ymax; g.ymax = p.ymax;
        g.zmin = -p.zmax; g.zmax = p.zmax;
        g.dcell = (g.xmax - g.xmin) / (double)g.nx;
    }
    {   // the band after the grid: an external field enters through the box
        const double box[3] = {g.xmax - g.xmin, g.ymax - g.ymin, g.zmax - g.zmin};
        if (!band_build(p, c->band, &why, c->species.thresholds(), box)) {
            delete c;
            return fail(nullptr, MOCHII_ERR_BAD_PARAM, why);
        }
    }
    c->fp32 = p.precision == MOCHII_PREC_FP32;
    c->tally64 = !c->fp32 || p.tally64;
    c->xscore = p.ion_add_dust || p.add_fuv;
    c->scatter = p.ion_add_dust && p.ion_dust_scatter;
    c->nabs = p.He_abund > 0.0 || c->xscore ? 4 : 1;
    c->ntally = c->xscore ? 8 : p.He_abund > 0.0 ? 6 : 2;
    if (p.ion_add_dust) {   // ion_dust_read (gas_opacity_mod.f90:69-121)
        if (!dust_table_read(p.ion_dust_kext, p.lambda_ref, c->dust_host, &why)) {
            delete c;
            return fail(nullptr, MOCHII_ERR_TABLE, why);
        }
        c->dust.n = (int)c->dust_host.lam.size();
    }
    c->nnu = c->band.nnu_band;
    const long long n = g.nleaf;
    auto bail = [&](int rc) {
        std::string m = c->last_error;
        release(c);
        delete c;
        return fail(nullptr, rc, m);
    };
#define CKI(call)                                                                         \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            c->last_error = std::string(#call) + ": " + cudaGetErrorString(e_);           \
            return bail(MOCHII_ERR_CUDA);                                                 \
        }                                                                                 \
    } while (0)
    CKI(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CKI(cudaEventCreate(&c->ev0));
    CKI(cudaEventCreate(&c->ev1));
    CKI(cudaEventCreate(&c->evA));
    CKI(cudaEventCreate(&c->evB));
    // leaf state (gas_state_setup, gas_state_mod.f90:58-77) on the host
    std::vector<double> nH(n, 1.0), xHI(n, p.xHI_init), xHeI(n, p.xHeI_init), xHeII(n, p.xHeII_init), ne(n),
        Te(n, p.te_fixed);
    if (!p.grid_car) {   // the file's n_H, then the namelist density model on the file's leaf centres
        for (long long il = 0; il < n; ++il) {
            nH[il] = lnH[il];
            if (p.nH_const >= 0.0) nH[il] = p.nH_const;   // grid_mod_amr.f90:137-147
            if (p.rmax > 0.0 || p.rmin > 0.0) {
                const double rho = std::sqrt(lx[il] * lx[il] + ly[il] * ly[il] + lz[il] * lz[il]);
                if (p.rmax > 0.0 && rho > p.rmax) nH[il] = 0.0;
                if (p.rmin > 0.0 && rho < p.rmin) nH[il] = 0.0;
            }
        }
        for (long long i = 0; i < n; ++i)
            ne[i] = nH[i] * ((1.0 - xHI[i]) + p.He_abund * (xHeII[i] + 2.0 * std::max(0.0, 1.0 - xHeI[i] - xHeII[i])));
    } else {
        const double dcx = 2.0 * p.xmax / p.nx, dcy = 2.0 * p.ymax / p.ny, dcz = 2.0 * p.zmax / p.nz;
        long long il = 0;
        for (int iz = 0; iz < p.nz; ++iz)
            for (int iy = 0; iy < p.ny; ++iy)
                for (int ix = 0; ix < p.nx; ++ix, ++il) {
                    if (p.nH_const >= 0.0) nH[il] = p.nH_const;   // grid_mod_amr.f90:137-147
                    if (p.rmax > 0.0 || p.rmin > 0.0) {
                        const double xl = -p.xmax + ((double)ix + 0.5) * dcx;
                        const double yl = -p.ymax + ((double)iy + 0.5) * dcy;
                        const double zl = -p.zmax + ((double)iz + 0.5) * dcz;
                        const double rho = std::sqrt(xl * xl + yl * yl + zl * zl);
                        if (p.rmax > 0.0 && rho > p.rmax) nH[il] = 0.0;
                        if (p.rmin > 0.0 && rho < p.rmin) nH[il] = 0.0;
                    }
                }
        for (long long i = 0; i < n; ++i)
            ne[i] = nH[i] * ((1.0 - xHI[i]) + p.He_abund * (xHeII[i] + 2.0 * std::max(0.0, 1.0 - xHeI[i] - xHeII[i])));
    }
    if (!p.grid_car || !p.car_walk_dda) {
        if (p.grid_car) {   // par%car_walk = 'amr': the car grid's walk tables
            car_walk_tables(g.nx, g.ny, g.nz, g.xmin, g.ymin, g.zmin, g.dcell, oh);
            c->lhalf.assign(n, 0.5 * g.dcell);
        }
        // the octree tables in one allocation: cell geo | children | leaf of cell | leaf geo | leaf faces
        const size_t nc = oh.ncells, nl = oh.nleaf;
        auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
        const size_t b_geo = al(nc * 32), b_ch = al(nc * 32), b_il = al(nc * 4), b_lg = al(nl * 32), b_ln = al(nl * 32);
        CKI(cudaMalloc(&c->oct_blob, b_geo + b_ch + b_il + b_lg + b_ln));
        char* base = static_cast<char*>(c->oct_blob);
        CKI(cudaMemcpy(base, oh.geo.data(), nc * 32, cudaMemcpyHostToDevice));
        CKI(cudaMemcpy(base + b_geo, oh.children.data(), nc * 32, cudaMemcpyHostToDevice));
        CKI(cudaMemcpy(base + b_geo + b_ch, oh.ileaf.data(), nc * 4, cudaMemcpyHostToDevice));
        CKI(cudaMemcpy(base + b_geo + b_ch + b_il, oh.lgeo.data(), nl * 32, cudaMemcpyHostToDevice));
        CKI(cudaMemcpy(base + b_geo + b_ch + b_il + b_lg, oh.lnext.data(), nl * 32, cudaMemcpyHostToDevice));
        c->oct.ncells = oh.ncells;
        c->oct.nshared = oh.nshared;
        c->oct.half = oh.half;
        c->oct.geo = reinterpret_cast<const double4*>(base);
        c->oct.children = reinterpret_cast<const int*>(base + b_geo);
        c->oct.ileaf = reinterpret_cast<const int*>(base + b_geo + b_ch);
        c->oct.lgeo = reinterpret_cast<const double4*>(base + b_geo + b_ch + b_il);
        c->oct.lnext = reinterpret_cast<const int*>(base + b_geo + b_ch + b_il + b_lg);
        if (p.grid_car) {
            c->oct.ncells = (int)n;   // no cell tables: every walk step stays on leaves
            c->oct.car = 1;
            c->oct.n[0] = g.nx; c->oct.n[1] = g.ny; c->oct.n[2] = g.nz;
            c->oct.org[0] = g.xmin; c->oct.org[1] = g.ymin; c->oct.org[2] = g.zmin;
            c->oct.hi[0] = g.xmax; c->oct.hi[1] = g.ymax; c->oct.hi[2] = g.zmax;
            c->oct.dcell = g.dcell;
        }
    }
    CKI(dalloc(&c->nH, n));
    CKI(dalloc(&c->xHI, n));
    CKI(dalloc(&c->xHeI, n));
    CKI(dalloc(&c->xHeII, n));
    CKI(dalloc(&c->ne, n));
    CKI(dalloc(&c->Te, n));
    CKI(cudaMemcpy(c->nH, nH.data(), n * 8, cudaMemcpyHostToDevice));
    CKI(cudaMemcpy(c->xHI, xHI.data(), n * 8, cudaMemcpyHostToDevice));
    CKI(cudaMemcpy(c->xHeI, xHeI.data(), n * 8, cudaMemcpyHostToDevice));
    CKI(cudaMemcpy(c->xHeII, xHeII.data(), n * 8, cudaMemcpyHostToDevice));
    CKI(cudaMemcpy(c->ne, ne.data(), n * 8, cudaMemcpyHostToDevice));
    CKI(cudaMemcpy(c->Te, Te.data(), n * 8, cudaMemcpyHostToDevice));
    const size_t rsz = c->fp32 ? 4 : 8;
    const size_t tsz = c->fp32 ? 8 : 8;   // float2 pair or double
    CKI(cudaMalloc(&c->col, (size_t)n * c->nabs * rsz + 64));
    CKI(cudaMalloc(&c->tally, (size_t)n * c->ntally * tsz + 64));
    CKI(cudaMalloc(&c->jt, (size_t)n * c->nnu * tsz + 64));
    CKI(dalloc(&c->rates, 8 * (size_t)n));   // gamma/heat of H I, He I, He II; heat_dust; G0
    CKI(cudaMemsetAsync(c->rates, 0, 8 * (size_t)n * 8, c->stream));
    if (c->dust.n > 0) {   // grey dust opacity per leaf, grid_mod_amr.f90:233-278 ('global_dgr' or 'none')
        std::vector<double> rk(n, 0.0);
        if (p.dust_law == 0)
            for (long long il = 0; il < n; ++il) rk[il] = nH[il] * p.cext_dust * p.DGR * p.distance2cm;
        CKI(dalloc(&c->rhokap, (size_t)n));
        CKI(cudaMemcpy(c->rhokap, rk.data(), n * 8, cudaMemcpyHostToDevice));
        const size_t nd = c->dust_host.lam.size();
        CKI(dalloc(&c->dust_blob, 4 * nd));
        CKI(cudaMemcpy(c->dust_blob, c->dust_host.lam.data(), nd * 8, cudaMemcpyHostToDevice));
        CKI(cudaMemcpy(c->dust_blob + nd, c->dust_host.alb.data(), nd * 8, cudaMemcpyHostToDevice));
        CKI(cudaMemcpy(c->dust_blob + 2 * nd, c->dust_host.gcos.data(), nd * 8, cudaMemcpyHostToDevice));
        CKI(cudaMemcpy(c->dust_blob + 3 * nd, c->dust_host.cext.data(), nd * 8, cudaMemcpyHostToDevice));
        c->dust.lam = c->dust_blob;
        c->dust.alb = c->dust_blob + nd;
        c->dust.gcos = c->dust_blob + 2 * nd;
        c->dust.cext = c->dust_blob + 3 * nd;
        c->dust.cref = c->dust_host.cref;
    }
    CKI(cudaMemset(c->rates, 0, 6 * (size_t)n * 8));
    if (!c->species.tr.empty()) {
        // registry tables in one blob: el | tr | st | photo | form | eth | lamref | Ssup
        const SpeciesHost& sp = c->species;
        MetalDev& m = c->metal;
        m.nel = (int)sp.el.size();
        m.ntr = (int)sp.tr.size();
        m.nst = (int)sp.st.size();
        m.ntrp = (m.ntr + 3) / 4 * 4;
        auto al = [](size_t b) { return (b + 255) / 256 * 256; };
        const size_t b_el = al(sp.el.size() * sizeof(MetalEl)), b_tr = al(sp.tr.size() * sizeof(MetalTr)),
                     b_st = al(sp.st.size() * sizeof(MetalStage)), b_ph = al(sp.photo.size() * 8),
                     b_fo = al(sp.form.size() * 4), b_et = al(sp.eth_flat.size() * 8), b_lr = al(sp.lamref.size() * 8),
                     b_ss = al(sp.Ssup.size() * 8);
        char* blob = nullptr;
        CKI(cudaMalloc(&blob, b_el + b_tr + b_st + b_ph + b_fo + b_et + b_lr + b_ss));
        char* q = blob;
        auto put = [&](const void* src, size_t bytes, size_t span) {
            char* dst = q;
            if (bytes) cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
            q += span;
            return dst;
        };
        m.el = reinterpret_cast<const MetalEl*>(put(sp.el.data(), sp.el.size() * sizeof(MetalEl), b_el));
        m.tr = reinterpret_cast<const MetalTr*>(put(sp.tr.data(), sp.tr.size() * sizeof(MetalTr), b_tr));
        m.st = reinterpret_cast<const MetalStage*>(put(sp.st.data(), sp.st.size() * sizeof(MetalStage), b_st));
        m.photo = reinterpret_cast<const double*>(put(sp.photo.data(), sp.photo.size() * 8, b_ph));
        m.form = reinterpret_cast<const int*>(put(sp.form.data(), sp.form.size() * 4, b_fo));
        m.eth = reinterpret_cast<const double*>(put(sp.eth_flat.data(), sp.eth_flat.size() * 8, b_et));
        m.lamref = reinterpret_cast<const double*>(put(sp.lamref.data(), sp.lamref.size() * 8, b_lr));
        m.Ssup = reinterpret_cast<const double*>(put(sp.Ssup.data(), sp.Ssup.size() * 8, b_ss));
        CKI(cudaGetLastError());
        if (sp.ntab > 0) {
            CKI(nl_log_tables(m.lamref, m.Ssup, sp.ntab, &c->metal_lnl, c->stream));
            m.lnL = c->metal_lnl;
        }
        CKI(dalloc(&m.egam, (size_t)n * m.ntr));
        CKI(dalloc(&m.eheat, (size_t)n * m.ntr));
        CKI(cudaMemset(m.egam, 0, (size_t)n * m.ntr * 8));
        CKI(cudaMemset(m.eheat, 0, (size_t)n * m.ntr * 8));
        CKI(cudaMalloc(&m.opac, (size_t)n * m.ntrp * rsz + 64));
        CKI(cudaMemset(m.opac, 0, (size_t)n * m.ntrp * rsz));
        if (p.metal_moments) {
            species_moment_tables(c->species, p.add_fuv ? p.efuv_min : p.eion_min, p.eion_max);
            const SpeciesHost& s2 = c->species;
            m.nmb = (int)s2.medge.size() - 1;
            // one allocation: medge | mcoef | mb0 | jof (element order of each threshold-order index)
            std::vector<int> jof(m.ntrp, -1);
            for (int j = 0; j < m.ntr; ++j) jof[s2.tr[j].flat] = j;
            const size_t b1 = al(s2.medge.size() * 8), b2 = al(s2.mcoef.size() * 8), b3 = al(s2.mb0.size() * 4),
                         b4 = al(jof.size() * 4);
            char* mq = nullptr;
            CKI(cudaMalloc(&mq, b1 + b2 + b3 + b4));
            CKI(cudaMemcpy(mq, s2.medge.data(), s2.medge.size() * 8, cudaMemcpyHostToDevice));
            CKI(cudaMemcpy(mq + b1, s2.mcoef.data(), s2.mcoef.size() * 8, cudaMemcpyHostToDevice));
            CKI(cudaMemcpy(mq + b1 + b2, s2.mb0.data(), s2.mb0.size() * 4, cudaMemcpyHostToDevice));
            CKI(cudaMemcpy(mq + b1 + b2 + b3, jof.data(), jof.size() * 4, cudaMemcpyHostToDevice));
            m.medge = reinterpret_cast<const double*>(mq);
            m.mcoef = reinterpret_cast<const double*>(mq + b1);
            m.mb0 = reinterpret_cast<const int*>(mq + b1 + b2);
            m.jof = reinterpret_cast<const int*>(mq + b1 + b2 + b3);
            m.mom32 = c->fp32 && c->tally64;
            CKI(cudaMalloc(&m.mom, mom_bytes(c) + 64));
        } else {
            m.raw32 = c->fp32 && c->tally64;
            CKI(cudaMalloc(&m.raw, raw_bytes(c) + 64));
        }
    }
    // sampler tables, component table, bin edges, QMC tables
    std::vector<double> te, tf, tc, comp;
    std::vector<int> off{0};
    for (int k = 0; k < c->band.ncomp; ++k) {
        const EnergyTable& t = c->band.tables[k];
        te.insert(te.end(), t.energy.begin(), t.energy.end());
        tf.insert(tf.end(), t.density.begin(), t.density.end());
        tc.insert(tc.end(), t.cdf.begin(), t.cdf.end());
        off.push_back((int)te.size());
        comp.push_back(c->band.comp_cdf[k]);
        comp.push_back(c->band.comp_x[k]);
        comp.push_back(c->band.comp_y[k]);
        comp.push_back(c->band.comp_z[k]);
    }
    CKI(dalloc(&c->tab.tab_e, te.size()));
    CKI(dalloc(&c->tab.tab_f, tf.size()));
    CKI(dalloc(&c->tab.tab_c, tc.size()));
    CKI(dalloc(&c->tab.tab_off, off.size()));
    CKI(dalloc(&c->tab.comp, comp.size()));
    CKI(dalloc(&c->tab.eedge, c->band.eedge.size()));
    CKI(dalloc(&c->tab.qmc, 1));
    CKI(cudaMemcpy(c->tab.tab_e, te.data(), te.size() * 8, cudaMemcpyHostToDevice));
    CKI(cudaMemcpy(c->tab.tab_f, tf.data(), tf.size() * 8, cudaMemcpyHostToDevice));
    CKI(cudaMemcpy(c->tab.tab_c, tc.data(), tc.size() * 8, cudaMemcpyHostToDevice));
    CKI(cudaMemcpy(c->tab.tab_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
    CKI(cudaMemcpy(c->tab.comp, comp.data(), comp.size() * 8, cudaMemcpyHostToDevice));
    CKI(cudaMemcpy(c->tab.eedge, c->band.eedge.data(), c->band.eedge.size() * 8, cudaMemcpyHostToDevice));
    QmcTables qt;
    qmc_build_tables(p.qmc_seed, qt);
    CKI(cudaMemcpy(c->tab.qmc, &qt, sizeof(qt), cudaMemcpyHostToDevice));
    // work areas
    c->tw.ledger_blocks = transport_blocks(c);
    CKI(dalloc(&c->tw.ledger, 3 * (size_t)c->tw.ledger_blocks));
    CKI(dalloc(&c->tw.counters, 4));
    if (c->band.slab) {   // slab_tally_setup (jtally_mod.f90:60-71)
        CKI(dalloc(&c->slab_iesc, 2 * (size_t)p.slab_nmu));
        CKI(cudaMemset(c->slab_iesc, 0, 2 * (size_t)p.slab_nmu * 8));
        c->slab_host.assign(2 * (size_t)p.slab_nmu, 0.0);
    }
    // packet records: launch chunks of up to 4 Mi packets
    CKI(alloc_records(c, std::min<long long>(p.nphotons, std::max<long long>(p.packet_chunk, 1024))));
    CKI(peel_setup(c));   // ion_peel_setup: observers and image plane (par%ion_peel)
    c->bw.blocks = balance_blocks(c);
    if (p.diffuse_field) {
        MilneHost mh;
        milne_tables_build(p.eion_max, mh);
        const size_t nt = mh.xg.size() + mh.cdf.size() + mh.xbar.size() + mh.frac.size();
        CKI(dalloc(&c->dif.tables, nt));
        double* q = c->dif.tables;
        CKI(cudaMemcpy(q, mh.xg.data(), mh.xg.size() * 8, cudaMemcpyHostToDevice));
        c->dif.m.xg = q;
        q += mh.xg.size();
        CKI(cudaMemcpy(q, mh.cdf.data(), mh.cdf.size() * 8, cudaMemcpyHostToDevice));
        c->dif.m.cdf = q;
        q += mh.cdf.size();
        CKI(cudaMemcpy(q, mh.xbar.data(), mh.xbar.size() * 8, cudaMemcpyHostToDevice));
        c->dif.m.xbar = q;
        q += mh.xbar.size();
        CKI(cudaMemcpy(q, mh.frac.data(), mh.frac.size() * 8, cudaMemcpyHostToDevice));
        c->dif.m.frac = q;
        c->dif.m.lgT0 = mh.lgT[0];
        c->dif.m.dlgT = mh.lgT[1] - mh.lgT[0];
        if (p.hei_diffuse) {   // main.f90:107-112: the He I excited channel's two-photon table
            std::string dir = p.data_dir;
            if (dir.empty()) {   // the directory above the atomic tables (<data_dir>/atomic)
                const std::string ad = atomic_dir(p);
                const size_t k = ad.find_last_of('/');
                dir = k == std::string::npos ? std::string(".") : ad.substr(0, k);
            }
            HeI2phHost hh;
            if (!hei_2ph_build(dir + "/HeI2phot.dat", p.eion_max, hh)) {
                c->last_error = "cannot read " + dir + "/HeI2phot.dat (par%data_dir)";
                return bail(MOCHII_ERR_TABLE);
            }
            CKI(dalloc(&c->dif.he_tab, 2 * (size_t)kHe2phN));
            CKI(cudaMemcpy(c->dif.he_tab, hh.cdf_e.data(), kHe2phN * 8, cudaMemcpyHostToDevice));
            CKI(cudaMemcpy(c->dif.he_tab + kHe2phN, hh.grid_y.data(), kHe2phN * 8, cudaMemcpyHostToDevice));
            c->dif.he.cdf_e = c->dif.he_tab;
            c->dif.he.grid_y = c->dif.he_tab + kHe2phN;
            c->dif.he.e_per_decay = hh.e_per_decay;
        }
        CKI(dalloc(&c->dif.ch, 4 * (size_t)n));
        CKI(dalloc(&c->dif.tot, (size_t)n));
        c->dif.scan_bytes = diffuse_scan_bytes(n);
        CKI(cudaMalloc(&c->dif.scan_tmp, c->dif.scan_bytes + 16));
    }
    if (p.solve_te) {
        ThermalHost th;
        if (!thermal_tables_build(p, th, &why)) {
            c->last_error = why;
            return bail(MOCHII_ERR_TABLE);
        }
        std::vector<double> tinv(kNlNT);
        for (int i = 0; i < kNlNT; ++i) tinv[i] = 1.0 / std::pow(10.0, 2.0 + 0.01 * (double)i);
        CKI(dalloc(&c->th.gff, (size_t)kGffNT * kGffNZ));
        CKI(cudaMemcpy(c->th.gff, th.gff, sizeof(th.gff), cudaMemcpyHostToDevice));
        CKI(dalloc(&c->th.tinv, (size_t)kNlNT));
        CKI(cudaMemcpy(c->th.tinv, tinv.data(), kNlNT * 8, cudaMemcpyHostToDevice));
        c->th.hi_nterm = th.hi_nterm;
        for (int i = 0; i < th.hi_nterm; ++i) { c->th.hi_A[i] = th.hi_A[i]; c->th.hi_T[i] = th.hi_T[i]; }
        c->th.use_hi_table = th.use_hi_table ? 1 : 0;
        if (th.use_hi_table) {
            CKI(dalloc(&c->th.lamref, (size_t)kNlNT));
            CKI(dalloc(&c->th.Ssup, (size_t)kNlNT * kNlNNE));
            CKI(cudaMemcpy(c->th.lamref, th.hi_lamref.data(), kNlNT * 8, cudaMemcpyHostToDevice));
            CKI(cudaMemcpy(c->th.Ssup, th.hi_Ssup.data(), (size_t)kNlNT * kNlNNE * 8, cudaMemcpyHostToDevice));
            CKI(nl_log_tables(c->th.lamref, c->th.Ssup, 1, &c->th.lnL, c->stream));
        }
        c->thermal_ready = true;
        if (c->metal.ntr > 0 && p.metal_rate_table) CKI(metal_ttable_build(c));
    }
    CKI(dalloc(&c->bw.partial, 6 * (size_t)c->bw.blocks));
    CKI(dalloc(&c->bw.counters, 8));
    CKI(launch_columns(c));
    CKI(cudaStreamSynchronize(c->stream));
    c->columns_fresh = true;
#undef CKI
    *out = c;
    return MOCHII_OK;
}

extern "C" void mochii_destroy(mochii_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    release(c);
    delete c;
}

// ---- batched nebulae -------------------------------------------------------
struct mochii_batch {
    std::vector<mochii_ctx*> ctx;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};   // per solve_te
    void* tb = nullptr;                             // the batched thermal solve
    bool batched_thermal = false;
    // pinned host copies the graph writes each iteration
    std::vector<double*> ledger;                    // 3 x ledger_blocks per nebula
    std::vector<unsigned long long*> tcount;        // 4 per nebula
    std::vector<double*> part;                      // 6 x balance blocks per nebula
    std::vector<unsigned long long*> bcount;        // 8 per nebula
    std::vector<uint64_t> gen;                      // each context's generation at mochii_batch_create
    mochii_mlp* mlp = nullptr;                      // the learned warm start recorded in the graph
    std::string err;
};

namespace {

// One nebula's pass into stream s, without synchronisation: the tally reset,
// the stellar transport, the rate normalisation, and copies of the ledger and
// counters to the batch's host buffers.
cudaError_t batch_pass(mochii_ctx* c, mochii_batch* b, int k, cudaStream_t s) {
    const long long n = c->grid.nleaf;
    const size_t tsz = 8;
    cudaError_t e;
    const cudaStream_t own = c->stream;
    c->stream = s;
    do {
        if ((e = cudaMemsetAsync(c->tally, 0, (size_t)n * c->ntally * tsz, s)) != cudaSuccess) break;
        if ((e = cudaMemsetAsync(c->jt, 0, (size_t)n * c->nnu * tsz, s)) != cudaSuccess) break;
        if (c->metal.ntr > 0 && c->metal.nmb > 0)
            e = cudaMemsetAsync(c->metal.mom, 0, mom_bytes(c), s);
        else if (c->metal.ntr > 0)
            e = cudaMemsetAsync(c->metal.raw, 0, raw_bytes(c), s);
        if (e != cudaSuccess) break;
        if ((e = cudaMemsetAsync(c->tw.counters, 0, 4 * sizeof(unsigned long long), s)) != cudaSuccess) break;
        if ((e = launch_transport(c)) != cudaSuccess) break;
        if ((e = launch_rates(c)) != cudaSuccess) break;
        if ((e = cudaMemcpyAsync(b->ledger[k], c->tw.ledger, 3 * (size_t)c->tw.ledger_blocks * 8, cudaMemcpyDeviceToHost,
                                 s)) != cudaSuccess)
            break;
        e = cudaMemcpyAsync(b->tcount[k], c->tw.counters, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    } while (false);
    c->stream = own;
    return e;
}

cudaError_t batch_record(mochii_batch* b, int solve_te, cudaGraphExec_t* out) {
    cudaError_t e = cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    const int n = (int)b->ctx.size();
    for (int k = 0; k < n && e == cudaSuccess; ++k) {
        e = batch_pass(b->ctx[k], b, k, b->s);
        // the learned warm start from this pass's rates (mochii_batch_set_warm_start)
        if (e == cudaSuccess && b->mlp && solve_te) e = mlp_warm_start_enqueue(b->ctx[k], b->mlp, b->s);
    }
    if (e == cudaSuccess) {
        if (solve_te && b->batched_thermal) {
            e = thermal_batch_enqueue(b->tb, b->ctx.data(), b->s);
        } else {
            for (int k = 0; k < n && e == cudaSuccess; ++k) {
                mochii_ctx* c = b->ctx[k];
                const cudaStream_t own = c->stream;
                c->stream = b->s;
                e = cudaMemsetAsync(c->bw.counters, 0, 8 * sizeof(unsigned long long), b->s);
                if (e == cudaSuccess) e = solve_te ? launch_thermal(c) : launch_balance(c);
                c->stream = own;
            }
        }
    }
    for (int k = 0; k < n && e == cudaSuccess; ++k) {
        mochii_ctx* c = b->ctx[k];
        e = cudaMemcpyAsync(b->part[k], c->bw.partial, 6 * (size_t)c->bw.blocks * 8, cudaMemcpyDeviceToHost, b->s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->bcount[k], c->bw.counters, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, b->s);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(b->s, &g);
    if (e == cudaSuccess) e = ee;
    if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, 0);
    if (g) cudaGraphDestroy(g);
    return e;
}

void batch_free(mochii_batch* b) {
    if (!b) return;
    if (b->s) cudaStreamSynchronize(b->s);
    for (cudaGraphExec_t& x : b->exec)
        if (x) cudaGraphExecDestroy(x);
    if (b->tb) thermal_batch_destroy(b->tb);
    for (auto* p : b->ledger) if (p) cudaFreeHost(p);
    for (auto* p : b->tcount) if (p) cudaFreeHost(p);
    for (auto* p : b->part) if (p) cudaFreeHost(p);
    for (auto* p : b->bcount) if (p) cudaFreeHost(p);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->s) cudaStreamDestroy(b->s);
    delete b;
}

}  // namespace

extern "C" int mochii_batch_create(mochii_ctx* const* ctxs, int n, mochii_batch** out) {
    if (!ctxs || n < 1 || !out) return fail(nullptr, MOCHII_ERR_BAD_PARAM, "mochii_batch_create: bad argument");
    *out = nullptr;
    for (int k = 0; k < n; ++k) {
        mochii_ctx* c = ctxs[k];
        if (!c) return fail(nullptr, MOCHII_ERR_BAD_PARAM, "mochii_batch_create: null context");
        if (c->par.diffuse_field)
            return fail(nullptr, MOCHII_ERR_UNSUPPORTED, "batched nebulae: par%diffuse_field must be off");
        if (c->band.slab)   // the slab's boundary tally is read back per standalone pass only
            return fail(nullptr, MOCHII_ERR_UNSUPPORTED, "batched nebulae: source_geometry='slab' is not batched");
        if (c->device != ctxs[0]->device)
            return fail(nullptr, MOCHII_ERR_BAD_PARAM, "batched nebulae: the contexts must share one device");
    }
    auto* b = new mochii_batch();
    b->ctx.assign(ctxs, ctxs + n);
    for (int k = 0; k < n; ++k) b->gen.push_back(ctxs[k]->generation);
    cudaError_t e = cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&b->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->e1);
    b->ledger.assign(n, nullptr);
    b->tcount.assign(n, nullptr);
    b->part.assign(n, nullptr);
    b->bcount.assign(n, nullptr);
    for (int k = 0; k < n && e == cudaSuccess; ++k) {
        mochii_ctx* c = ctxs[k];
        e = cudaMallocHost(&b->ledger[k], 3 * (size_t)c->tw.ledger_blocks * 8);
        if (e == cudaSuccess) e = cudaMallocHost(&b->tcount[k], 4 * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMallocHost(&b->part[k], 6 * (size_t)c->bw.blocks * 8);
        if (e == cudaSuccess) e = cudaMallocHost(&b->bcount[k], 8 * sizeof(unsigned long long));
        // the state the first recorded pass reads must be on the device
        if (e == cudaSuccess && !c->columns_fresh) {
            e = launch_columns(c);
            c->columns_fresh = true;
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    }
    bool all = true;
    for (int k = 0; k < n; ++k) {
        const mochii_ctx* c = ctxs[k];
        all = all && c->metal.ntr > 0 && c->par.solver_bracketed && c->thermal_ready &&
              (c->par.solver_warp == 0 || c->par.solver_warp == 3) && c->par.solver_warp == ctxs[0]->par.solver_warp;
    }
    if (e == cudaSuccess && all) {
        b->tb = thermal_batch_create(ctxs, n, &e);
        b->batched_thermal = b->tb != nullptr;
    }
    if (e != cudaSuccess) {
        const std::string m = std::string("mochii_batch_create: ") + cudaGetErrorString(e);
        batch_free(b);
        return fail(nullptr, MOCHII_ERR_CUDA, m);
    }
    *out = b;
    return MOCHII_OK;
}

extern "C" int mochii_batch_iterate(mochii_batch* b, int solve_te, mochii_pass_stats* st, mochii_metrics* mm,
                                    double* device_ms) {
    if (!b) return MOCHII_ERR_BAD_PARAM;
    const int n = (int)b->ctx.size();
    const int slot = solve_te ? 1 : 0;
    for (int k = 0; k < n; ++k) {
        mochii_ctx* c = b->ctx[k];
        if (solve_te && !c->thermal_ready)
            return fail(c, MOCHII_ERR_BAD_PARAM, "the thermal solve needs par%solve_te = .true. at mochii_init");
        // the recorded graph holds this context's launch shapes and buffers
        if (c->generation != b->gen[k])
            return fail(c, MOCHII_ERR_BAD_PARAM,
                        "a batched context's parameters or tuning changed after mochii_batch_create; create a new batch");
    }
    cudaError_t e = cudaSuccess;
    for (mochii_ctx* c : b->ctx) {   // the contexts' own work first
        if (!c->columns_fresh) {
            e = launch_columns(c);
            c->columns_fresh = true;
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return fail(c, MOCHII_ERR_CUDA, cudaGetErrorString(e));
    }
    if (!b->exec[slot] && (e = batch_record(b, solve_te, &b->exec[slot])) != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, MOCHII_ERR_CUDA, std::string("recording the batch graph: ") + cudaGetErrorString(e));
    }
    e = cudaEventRecord(b->e0, b->s);
    if (e == cudaSuccess) e = cudaGraphLaunch(b->exec[slot], b->s);
    if (e == cudaSuccess) e = cudaEventRecord(b->e1, b->s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->s);
    if (e != cudaSuccess) return fail(nullptr, MOCHII_ERR_CUDA, cudaGetErrorString(e));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->e0, b->e1);
    if (device_ms) *device_ms = ms;
    int status = MOCHII_OK;
    for (int k = 0; k < n; ++k) {
        mochii_ctx* c = b->ctx[k];
        c->columns_fresh = true;
        mochii_pass_stats s;
        std::memset(&s, 0, sizeof(s));
        long double en[3] = {0, 0, 0};
        for (int q = 0; q < c->tw.ledger_blocks; ++q)
            for (int j = 0; j < 3; ++j) en[j] += (long double)b->ledger[k][3 * (size_t)q + j];
        s.energy_emitted = (double)en[0];
        s.energy_absorbed = (double)en[1];
        s.energy_escaped = (double)en[2];
        s.closure = std::fabs(s.energy_absorbed + s.energy_escaped - s.energy_emitted) / std::max(s.energy_emitted, kTinest);
        s.direct_segments = (int64_t)b->tcount[k][0];
        s.walk_kills = (int64_t)b->tcount[k][1];
        s.metal_active = (int64_t)b->tcount[k][2];
        s.scattered_segments = (int64_t)b->tcount[k][3];
        s.packets = c->par.nphotons;
        c->last_pass = s;
        if (st) st[k] = s;
        mochii_metrics r;
        std::memset(&r, 0, sizeof(r));
        const double* q = b->part[k];
        if (solve_te) {
            double sm[4] = {0, 0, 0, 0};
            for (int bl = 0; bl < c->bw.blocks; ++bl) {
                r.max_dx = std::max(r.max_dx, q[6 * (size_t)bl]);
                r.max_dte = std::max(r.max_dte, q[6 * (size_t)bl + 1]);
                for (int j = 0; j < 4; ++j) sm[j] += q[6 * (size_t)bl + 2 + j];
            }
            r.dx_vol = sm[0] / std::max(sm[1], kTinest);
            r.dte_vol = sm[2] / std::max(sm[3], kTinest);
        } else {
            double sdx = 0.0, sx = 0.0;
            for (int bl = 0; bl < c->bw.blocks; ++bl) {
                r.max_dx = std::max(r.max_dx, q[3 * (size_t)bl]);
                sdx += q[3 * (size_t)bl + 1];
                sx += q[3 * (size_t)bl + 2];
            }
            r.dx_vol = sdx / std::max(sx, kTinest);
        }
        const unsigned long long* cnt = b->bcount[k];
        r.cells_solved = (int64_t)cnt[0];
        r.fixed_point_cap_hits = (int64_t)cnt[1];
        r.fixed_point_passes = (int64_t)cnt[2];
        r.metal_sum_calls = (int64_t)cnt[3];
        r.rate_evaluations = (int64_t)cnt[4];
        r.warm_accepted = (int64_t)cnt[5];
        if (mm) mm[k] = r;
        if (!std::isfinite(s.energy_emitted) || !std::isfinite(s.energy_absorbed)) {
            status = fail(c, MOCHII_ERR_NONFINITE, "non-finite energy ledger");
        } else if (s.closure > 5.0e-13) {
            status = fail(c, MOCHII_ERR_CLOSURE, "energy closure exceeds 5e-13");
        }
    }
    return status;
}

extern "C" int mochii_batch_set_warm_start(mochii_batch* b, mochii_mlp* m) {
    if (!b || !m) return MOCHII_ERR_BAD_PARAM;
    if (!b->batched_thermal)
        return fail(nullptr, MOCHII_ERR_UNSUPPORTED,
                    "the batch warm start needs the batched thermal solve (metals, thermal_solver 'bracketed', "
                    "cell_layout 'lane' or 'lockstep')");
    const int n = (int)b->ctx.size();
    double fac = 1.05;
    int rc = mlp_batch_prepare(m, b->ctx.data(), n, &fac);
    if (rc) return fail(nullptr, rc, "preparing the warm start for the batch");
    std::vector<double> facs(n, fac);
    cudaError_t e = thermal_batch_set_warm(b->tb, b->ctx.data(), facs.data(), 1.0e-6);
    if (e != cudaSuccess) return fail(nullptr, MOCHII_ERR_CUDA, cudaGetErrorString(e));
    for (int k = 0; k < n; ++k) b->gen[k] = b->ctx[k]->generation;   // the new warm-start arrays are the batch's own
    for (cudaGraphExec_t& x : b->exec)   // recorded again, now with the inference
        if (x) {
            cudaGraphExecDestroy(x);
            x = nullptr;
        }
    b->mlp = m;
    return MOCHII_OK;
}

extern "C" void mochii_batch_destroy(mochii_batch* b) { batch_free(b); }

extern "C" int64_t mochii_nleaf(const mochii_ctx* c) { return c ? c->grid.nleaf : 0; }
extern "C" int mochii_metal_shape(const mochii_ctx* c, int* ntransitions, int* nstages) {
    if (!c) return MOCHII_ERR_BAD_PARAM;
    if (ntransitions) *ntransitions = c->metal.ntr;
    if (nstages) *nstages = c->metal.nst;
    return MOCHII_OK;
}
extern "C" int mochii_nnu_band(const mochii_ctx* c) { return c ? c->nnu : 0; }
extern "C" double mochii_ion_Ltot(const mochii_ctx* c) { return c ? c->band.ion_Ltot : 0.0; }

extern "C" int mochii_set_nphotons(mochii_ctx* c, int64_t np) {
    if (!c || np < 1) return MOCHII_ERR_BAD_PARAM;
    ++c->generation;
    c->par.nphotons = np;
    const int nb = transport_blocks(c);
    if (nb > c->tw.ledger_blocks) {
        cudaFree(c->tw.ledger);
        c->tw.ledger = nullptr;
        CK(c, dalloc(&c->tw.ledger, 3 * (size_t)nb));
    }
    c->tw.ledger_blocks = nb;
    const long long cap = std::min<long long>(np, std::max<long long>(c->par.packet_chunk, 1024));
    if (cap > c->rec.cap) {
        CK(c, cudaStreamSynchronize(c->stream));
        free_records(c);
        CK(c, alloc_records(c, cap));
    }
    return MOCHII_OK;
}

// ionizing_field_and_rates, ionizing_field_mod.f90:72-170.
extern "C" int mochii_transport_pass(mochii_ctx* c, int with_peel, mochii_pass_stats* st) {
    if (!c) return MOCHII_ERR_BAD_PARAM;
    if (with_peel && !c->par.ion_peel)
        return fail(c, MOCHII_ERR_BAD_PARAM, "with_peel needs par%ion_peel = .true. at mochii_init (the observers)");
    if (with_peel) CK(c, peel_clear(c));
    c->peeling = with_peel != 0;   // the walk kernels peel every packet toward the observers
    struct PeelEnd {
        mochii_ctx* c;
        ~PeelEnd() { c->peeling = false; }
    } peel_end{c};
    const long long n = c->grid.nleaf;
    const size_t tsz = 8;
    if (!c->columns_fresh) {
        CK(c, launch_columns(c));
        c->columns_fresh = true;
    }
    CK(c, cudaEventRecord(c->evA, c->stream));
    // jt_ion(:,:) = 0 and ion_score_reset (ionizing_field_mod.f90:90-91)
    CK(c, cudaMemsetAsync(c->tally, 0, (size_t)n * c->ntally * tsz, c->stream));
    CK(c, cudaMemsetAsync(c->jt, 0, (size_t)n * c->nnu * tsz, c->stream));
    if (c->metal.ntr > 0 && c->metal.nmb > 0)   // species_rate_path_reset (species_mod.f90:321-326)
        CK(c, cudaMemsetAsync(c->metal.mom, 0, mom_bytes(c), c->stream));
    else if (c->metal.ntr > 0)
        CK(c, cudaMemsetAsync(c->metal.raw, 0, raw_bytes(c), c->stream));
    CK(c, cudaMemsetAsync(c->tw.counters, 0, 4 * sizeof(unsigned long long), c->stream));
    if (c->slab_iesc) CK(c, cudaMemsetAsync(c->slab_iesc, 0, c->slab_host.size() * 8, c->stream));
    CK(c, cudaEventRecord(c->ev0, c->stream));
    CK(c, launch_transport(c));
    double dlum = 0.0;
    long long nd = 0;
    if (c->par.diffuse_field) {   // ionizing_field_mod.f90:139-161
        CK(c, diffuse_build(c, &dlum));
        const double lpacket = c->band.ion_Ltot / (double)c->par.nphotons;
        nd = dlum > 0.0 ? std::llround(dlum / lpacket) : 0;
        if (nd > 0) CK(c, launch_transport_diffuse(c, dlum, nd));
    }
    CK(c, cudaEventRecord(c->ev1, c->stream));
    CK(c, launch_rates(c));
    CK(c, cudaEventRecord(c->evB, c->stream));
    std::vector<double> led(3 * (size_t)c->tw.ledger_blocks);
    unsigned long long cnt[4];
    CK(c, cudaMemcpyAsync(led.data(), c->tw.ledger, led.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaMemcpyAsync(cnt, c->tw.counters, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
    if (c->slab_iesc)
        CK(c, cudaMemcpyAsync(c->slab_host.data(), c->slab_iesc, c->slab_host.size() * 8, cudaMemcpyDeviceToHost,
                              c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    float ms = 0.0f, pms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    cudaEventElapsedTime(&pms, c->evA, c->evB);
    long double e[3] = {0, 0, 0};
    for (int b = 0; b < c->tw.ledger_blocks; ++b)
        for (int k = 0; k < 3; ++k) e[k] += (long double)led[3 * (size_t)b + k];
    mochii_pass_stats s;
    std::memset(&s, 0, sizeof(s));
    s.energy_emitted = (double)e[0];
    s.energy_absorbed = (double)e[1];
    s.energy_escaped = (double)e[2];
    s.closure = std::fabs(s.energy_absorbed + s.energy_escaped - s.energy_emitted) /
                std::max(s.energy_emitted, kTinest);
    s.direct_segments = (int64_t)cnt[0];
    s.scattered_segments = (int64_t)cnt[3];
    s.walk_kills = (int64_t)cnt[1];
    s.metal_active = (int64_t)cnt[2];
    s.kernel_ms = ms;
    s.pass_ms = pms;
    s.diffuse_packets = nd;
    s.diffuse_lum = dlum;
    s.packets = c->par.nphotons + nd;
    c->last_pass = s;
    if (st) *st = s;
    if (!std::isfinite(s.energy_emitted) || !std::isfinite(s.energy_absorbed))
        return fail(c, MOCHII_ERR_NONFINITE, "non-finite energy ledger");
    if (s.closure > 5.0e-13)   // ion_score_mod.f90:386
        return fail(c, MOCHII_ERR_CLOSURE, "energy closure exceeds 5e-13");
    return MOCHII_OK;
}

// gas_equilibrium_update (ion_balance_mod.f90:352) / gas_thermal_update
// (thermal_mod.f90:124).
extern "C" int mochii_balance_update(mochii_ctx* c, int solve_te, mochii_metrics* m) {
    if (!c) return MOCHII_ERR_BAD_PARAM;
    if (solve_te && !c->thermal_ready)
        return fail(c, MOCHII_ERR_BAD_PARAM, "the thermal solve needs par%solve_te = .true. at mochii_init (tables)");
    CK(c, cudaMemsetAsync(c->bw.counters, 0, 8 * sizeof(unsigned long long), c->stream));
    CK(c, cudaEventRecord(c->ev0, c->stream));
    if (solve_te) CK(c, launch_thermal(c));
    else CK(c, launch_balance(c));
    CK(c, cudaEventRecord(c->ev1, c->stream));
    // how far the solved T_e landed from a learned warm start: the first
    // bracketing step of the next one
    const bool learned = solve_te && c->twarm_set && c->twarm_learned;
    double werr[2] = {0.0, 0.0};
    if (learned) CK(c, warm_error_launch(c));
    c->twarm_set = false;
    c->twarm_learned = false;
    c->columns_fresh = true;   // both kernels refresh the columns they change
    const int np = solve_te ? 6 : 3;
    std::vector<double> part((size_t)np * c->bw.blocks);
    unsigned long long cnt[8];
    CK(c, cudaMemcpyAsync(part.data(), c->bw.partial, part.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaMemcpyAsync(cnt, c->bw.counters, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
    if (learned) CK(c, cudaMemcpyAsync(werr, c->twarm_err, sizeof(werr), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    if (learned && werr[1] >= 64.0) c->warm_err_ln = std::sqrt(werr[0] / werr[1]);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    mochii_metrics r;
    std::memset(&r, 0, sizeof(r));
    if (solve_te) {
        double s[4] = {0, 0, 0, 0};
        for (int b = 0; b < c->bw.blocks; ++b) {
            const double* q = &part[6 * (size_t)b];
            r.max_dx = std::max(r.max_dx, q[0]);
            r.max_dte = std::max(r.max_dte, q[1]);
            for (int k = 0; k < 4; ++k) s[k] += q[2 + k];
        }
        r.dx_vol = s[0] / std::max(s[1], kTinest);    // thermal_mod.f90:223-224
        r.dte_vol = s[2] / std::max(s[3], kTinest);
    } else {
        double sdx = 0.0, sx = 0.0;
        for (int b = 0; b < c->bw.blocks; ++b) {
            r.max_dx = std::max(r.max_dx, part[3 * (size_t)b]);
            sdx += part[3 * (size_t)b + 1];
            sx += part[3 * (size_t)b + 2];
        }
        r.dx_vol = sdx / std::max(sx, kTinest);
    }
    r.cells_solved = (int64_t)cnt[0];
    r.fixed_point_cap_hits = (int64_t)cnt[1];
    r.fixed_point_passes = (int64_t)cnt[2];
    r.metal_sum_calls = (int64_t)cnt[3];
    r.rate_evaluations = (int64_t)cnt[4];
    r.warm_accepted = (int64_t)cnt[5];
    r.kernel_ms = ms;
    if (m) *m = r;
    if (!std::isfinite(r.max_dx) || !std::isfinite(r.dx_vol) || !std::isfinite(r.max_dte))
        return fail(c, MOCHII_ERR_NONFINITE, "non-finite state after the solve");
    return MOCHII_OK;
}

// gas_opacity_fill (gas_opacity_mod.f90:299-332).  The balance kernel
// already rewrites the columns of every leaf it solves, so this launches
// only when the state changed through mochii_set_field since.
extern "C" int mochii_opacity_fill(mochii_ctx* c) {
    if (!c) return MOCHII_ERR_BAD_PARAM;
    if (c->columns_fresh) return MOCHII_OK;
    CK(c, launch_columns(c));
    CK(c, cudaStreamSynchronize(c->stream));
    c->columns_fresh = true;
    return MOCHII_OK;
}

namespace {
std::map<std::string, Tuning>& tune_cache() {
    static std::map<std::string, Tuning> m;
    return m;
}
std::string tune_key(const mochii_ctx* c) {
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, c->device);
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s|%dx%dx%d|%lld|%d|%d|%d|%d", prop.name, c->grid.nx, c->grid.ny, c->grid.nz,
                  c->grid.nleaf, c->fp32 ? 32 : 64, c->nabs, c->nnu, c->metal.ntr);
    return buf;
}
}  // namespace

extern "C" int mochii_set_tuning(mochii_ctx* c, const mochii_tuning* t) {
    if (!c || !t || t->lookahead < 0 || t->lookahead > 2 || t->walk_blocks_per_sm < 1 || t->walk_blocks_per_sm > 64 ||
        t->lane_threads < 0 || t->lane_threads % 32 != 0 || t->lane_threads > 1024)
        return fail(c, MOCHII_ERR_BAD_PARAM,
                    "tuning out of range (lookahead 0..2, blocks per SM 1..64, lane threads a multiple of 32)");
    ++c->generation;
    c->tune.lookahead = t->lookahead;
    c->tune.walk_blocks_per_sm = t->walk_blocks_per_sm;
    if (t->lane_threads != c->tune.lane_threads) {
        c->tune.lane_threads = t->lane_threads;
        c->bw.lane_threads = 0;   // the lane kernel's launch shape is rebuilt at the next thermal update
    }
    const int nb = transport_blocks(c);
    if (nb > c->tw.ledger_blocks) {
        cudaFree(c->tw.ledger);
        c->tw.ledger = nullptr;
        CK(c, dalloc(&c->tw.ledger, 3 * (size_t)nb));
    }
    c->tw.ledger_blocks = nb;
    return MOCHII_OK;
}

extern "C" int mochii_get_tuning(const mochii_ctx* c, mochii_tuning* t) {
    if (!c || !t) return MOCHII_ERR_BAD_PARAM;
    t->lookahead = c->tune.lookahead;
    t->walk_blocks_per_sm = c->tune.walk_blocks_per_sm;
    t->best_ms = c->tune.best_ms;
    t->lane_threads = c->tune.lane_threads;
    t->thermal_ms = c->tune.thermal_ms;
    return MOCHII_OK;
}

extern "C" int mochii_autotune(mochii_ctx* c, int64_t sample, mochii_tuning* out) {
    if (!c || sample < 1) return MOCHII_ERR_BAD_PARAM;
    const std::string key = tune_key(c);
    auto it = tune_cache().find(key);
    if (it != tune_cache().end()) {
        const Tuning cached = it->second;
        mochii_tuning t{cached.lookahead, cached.walk_blocks_per_sm, cached.best_ms, cached.lane_threads,
                        cached.thermal_ms};
        int rc = mochii_set_tuning(c, &t);
        c->tune = cached;
        if (out) *out = t;
        return rc;
    }
    const int64_t keep = c->par.nphotons;
    int rc = mochii_set_nphotons(c, std::min<int64_t>(sample, keep));
    if (rc) return rc;
    double best = 1e300;
    mochii_tuning bt{2, 8, 0.0, 0, 0.0};
    for (int la = 0; la <= 2; ++la)
        for (int bps : {4, 8, 16, 32}) {
            mochii_tuning t{la, bps, 0.0, c->tune.lane_threads, 0.0};
            if ((rc = mochii_set_tuning(c, &t))) return rc;
            double ms = 0.0;
            for (int rep = 0; rep < 3; ++rep) {
                mochii_pass_stats st;
                if ((rc = mochii_transport_pass(c, 0, &st))) return rc;
                if (rep > 0) ms += st.kernel_ms;   // first pass warms the variant
            }
            if (ms < best) { best = ms; bt = t; }
        }
    bt.best_ms = best / 2.0;
    if ((rc = mochii_set_tuning(c, &bt))) return rc;
    c->tune.best_ms = bt.best_ms;
    // the cell tile of the per-lane thermal solve: trial updates on the rates
    // of the last trial pass, each from the saved state, the state restored
    if (c->thermal_ready && c->metal.ntr > 0 && c->par.solver_bracketed && c->par.solver_warp == 3) {
        const long long n = c->grid.nleaf;
        double* save = nullptr;
        CK(c, cudaMalloc(&save, (size_t)5 * n * 8));
        double* fields[5] = {c->xHI, c->xHeI, c->xHeII, c->ne, c->Te};
        auto copy = [&](bool to_save) -> cudaError_t {
            for (int f = 0; f < 5; ++f) {
                cudaError_t e = to_save ? cudaMemcpyAsync(save + f * n, fields[f], n * 8, cudaMemcpyDeviceToDevice, c->stream)
                                        : cudaMemcpyAsync(fields[f], save + f * n, n * 8, cudaMemcpyDeviceToDevice, c->stream);
                if (e != cudaSuccess) return e;
            }
            return cudaSuccess;
        };
        cudaError_t e = copy(true);
        int best_threads = 0;
        double best_t = 1e300;
        for (int threads : {0, 192, 160, 128, 96}) {   // 0: the most lanes the rate cache fits
            if (e != cudaSuccess) break;
            c->tune.lane_threads = threads;
            c->bw.lane_threads = 0;
            double ms = 0.0;
            for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {
                if ((e = copy(false)) != cudaSuccess) break;
                mochii_metrics m;
                c->twarm_set = false;
                const int r2 = mochii_balance_update(c, 1, &m);
                if (r2) { cudaFree(save); return r2; }
                if (rep > 0) ms = m.kernel_ms;   // the first update warms the shape
            }
            if (e == cudaSuccess && ms < best_t) { best_t = ms; best_threads = threads; }
        }
        if (e == cudaSuccess) e = copy(false);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        cudaFree(save);
        CK(c, e);
        c->tune.lane_threads = best_threads;
        c->bw.lane_threads = 0;
        c->tune.thermal_ms = best_t;
        bt.lane_threads = best_threads;
        bt.thermal_ms = best_t;
        c->columns_fresh = false;   // the trial updates rewrote the columns
    }
    c->tune.tuned = true;
    tune_cache()[key] = c->tune;
    if ((rc = mochii_set_nphotons(c, keep))) return rc;
    if (out) *out = bt;
    return MOCHII_OK;
}

namespace {
double* field_ptr(mochii_ctx* c, const std::string& n, long long* count) {
    const long long nl = c->grid.nleaf;
    *count = nl;
    if (n == "nH") return c->nH;
    if (n == "x_HI") return c->xHI;
    if (n == "x_HeI") return c->xHeI;
    if (n == "x_HeII") return c->xHeII;
    if (n == "n_e") return c->ne;
    if (n == "T_e") return c->Te;
    static const char* rn[8] = {"gamma_HI", "gamma_HeI", "gamma_HeII", "heat_HI", "heat_HeI", "heat_HeII",
                                "heat_dust", "g0_fuv"};
    for (int k = 0; k < 8; ++k)
        if (n == rn[k]) return c->rates + (size_t)k * nl;
    if (n == "rhokap") return c->rhokap;   // null (no such field) without grains
    return nullptr;
}
}  // namespace

extern "C" int mochii_get_field(mochii_ctx* c, const char* name, double* out, int64_t n) {
    if (!c || !name || !out) return MOCHII_ERR_BAD_PARAM;
    const std::string nm(name);
    if (nm == "eedge") {
        if (n != (int64_t)c->band.eedge.size()) return fail(c, MOCHII_ERR_BAD_PARAM, "eedge size mismatch");
        std::memcpy(out, c->band.eedge.data(), n * 8);
        return MOCHII_OK;
    }
    if (nm == "T_dust") {   // dust_temp_compute (dust_temp_mod.f90:137-170) from the last pass's Heat_dust
        if (n != c->grid.nleaf) return fail(c, MOCHII_ERR_BAD_PARAM, "T_dust size mismatch");
        if (!c->par.ion_add_dust || !c->rhokap) return fail(c, MOCHII_ERR_BAD_PARAM, "T_dust: needs par%ion_add_dust");
        CK(c, dust_temp_launch(c));
        CK(c, cudaMemcpyAsync(out, c->tdust, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
        CK(c, cudaStreamSynchronize(c->stream));
        return MOCHII_OK;
    }
    if (nm == "T_warm") {   // the warm start of the next bracketed thermal solve, as set or predicted
        if (n != c->grid.nleaf) return fail(c, MOCHII_ERR_BAD_PARAM, "T_warm size mismatch");
        if (!c->twarm_set) return fail(c, MOCHII_ERR_BAD_PARAM, "T_warm: no warm start is set");
        CK(c, cudaMemcpyAsync(out, c->twarm, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
        CK(c, cudaStreamSynchronize(c->stream));
        return MOCHII_OK;
    }
    if (nm == "leaf_half") {
        if (n != c->grid.nleaf) return fail(c, MOCHII_ERR_BAD_PARAM, "leaf_half size mismatch");
        if (c->oct.ncells > 0) std::memcpy(out, c->lhalf.data(), n * 8);
        else for (int64_t i = 0; i < n; ++i) out[i] = 0.5 * c->grid.dcell;
        return MOCHII_OK;
    }
    if (nm == "gamma_metal" || nm == "heat_metal" || nm == "x_metal") {
        // leaf-major blocks in registry order: transitions (Gamma, heating) or
        // stages (fractions of the written state, species_write)
        if (c->metal.ntr == 0) return fail(c, MOCHII_ERR_BAD_PARAM, nm + ": par%use_metals is off");
        const long long per = nm == "x_metal" ? c->metal.nst : c->metal.ntr;
        const long long cnt = c->grid.nleaf * per;
        if (n != cnt) return fail(c, MOCHII_ERR_BAD_PARAM, nm + " size mismatch (nleaf*" + std::to_string(per) + ")");
        if (nm == "x_metal") {
            double* d = nullptr;
            CK(c, cudaMallocAsync(&d, cnt * 8, c->stream));
            CK(c, launch_metal_fractions(c, d));
            CK(c, cudaMemcpyAsync(out, d, cnt * 8, cudaMemcpyDeviceToHost, c->stream));
            CK(c, cudaFreeAsync(d, c->stream));
        } else {
            CK(c, cudaMemcpyAsync(out, nm == "gamma_metal" ? c->metal.egam : c->metal.eheat, cnt * 8,
                                  cudaMemcpyDeviceToHost, c->stream));
        }
        CK(c, cudaStreamSynchronize(c->stream));
        return MOCHII_OK;
    }
    if (nm == "jt_ion") {
        const long long cnt = c->grid.nleaf * (long long)c->nnu;
        if (n != cnt) return fail(c, MOCHII_ERR_BAD_PARAM, "jt_ion size mismatch (nleaf*nnu_band)");
        double* d = nullptr;
        CK(c, cudaMallocAsync(&d, cnt * 8, c->stream));
        CK(c, launch_jt_export(c, d));
        CK(c, cudaMemcpyAsync(out, d, cnt * 8, cudaMemcpyDeviceToHost, c->stream));
        CK(c, cudaFreeAsync(d, c->stream));
        CK(c, cudaStreamSynchronize(c->stream));
        return MOCHII_OK;
    }
    long long cnt = 0;
    double* p = field_ptr(c, nm, &cnt);
    if (!p) return fail(c, MOCHII_ERR_BAD_PARAM, "unknown field " + nm);
    if (n != cnt) return fail(c, MOCHII_ERR_BAD_PARAM, "size mismatch for " + nm);
    CK(c, cudaMemcpyAsync(out, p, cnt * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return MOCHII_OK;
}

extern "C" int mochii_set_field(mochii_ctx* c, const char* name, const double* in, int64_t n) {
    if (!c || !name || !in) return MOCHII_ERR_BAD_PARAM;
    const std::string nm(name);
    if (nm == "T_warm") {   // warm start of the next bracketed thermal solve
        if (n != c->grid.nleaf) return fail(c, MOCHII_ERR_BAD_PARAM, "size mismatch for T_warm");
        if (!c->twarm) {
            ++c->generation;
            CK(c, dalloc(&c->twarm, (size_t)n));
        }
        CK(c, cudaMemcpyAsync(c->twarm, in, n * 8, cudaMemcpyHostToDevice, c->stream));
        c->twarm_fac = 1.05;   // a caller's warm start: the default first step, no gate
        c->twarm_gate = 0.0;
        c->twarm_learned = false;
        CK(c, cudaStreamSynchronize(c->stream));
        c->twarm_set = true;
        return MOCHII_OK;
    }
    if (nm != "nH" && nm != "x_HI" && nm != "x_HeI" && nm != "x_HeII" && nm != "n_e" && nm != "T_e")
        return fail(c, MOCHII_ERR_BAD_PARAM, "field is not settable: " + nm);
    long long cnt = 0;
    double* p = field_ptr(c, nm, &cnt);
    if (n != cnt) return fail(c, MOCHII_ERR_BAD_PARAM, "size mismatch for " + nm);
    CK(c, cudaMemcpyAsync(p, in, cnt * 8, cudaMemcpyHostToDevice, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    c->columns_fresh = false;
    return MOCHII_OK;
}

extern "C" int mochii_sobol_uniforms(int seed, int stream, int64_t idx0, int64_t n, int nd, double* out) {
    if (!out || nd < 1 || nd > kQmcMaxDim || (stream != 1 && stream != 2) || n < 0 || idx0 < 0)
        return fail(nullptr, MOCHII_ERR_BAD_PARAM, "mochii_sobol_uniforms: bad argument");
    if (n == 0) return MOCHII_OK;
    QmcTables qt;
    qmc_build_tables(seed, qt);
    QmcTables* dq = nullptr;
    double* d = nullptr;
    cudaStream_t s = nullptr;
    auto cleanup = [&]() {
        if (dq) cudaFree(dq);
        if (d) cudaFree(d);
        if (s) cudaStreamDestroy(s);
    };
#define CKS(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) {                                                                         \
            cleanup();                                                                                   \
            return fail(nullptr, MOCHII_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
        }                                                                                                \
    } while (0)
    CKS(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CKS(cudaMalloc(&dq, sizeof(QmcTables)));
    CKS(cudaMalloc(&d, (size_t)n * nd * 8));
    CKS(cudaMemcpyAsync(dq, &qt, sizeof(qt), cudaMemcpyHostToDevice, s));
    CKS(launch_sobol(dq, stream - 1, idx0, n, nd, d, s));
    CKS(cudaMemcpyAsync(out, d, (size_t)n * nd * 8, cudaMemcpyDeviceToHost, s));
    CKS(cudaStreamSynchronize(s));
#undef CKS
    cleanup();
    return MOCHII_OK;
}

extern "C" int mochii_philox_uniforms(int64_t seed, int stream, int64_t packet, int n0, int n, double* out) {
    if (!out || n < 0 || n0 < 0 || packet < 0 || (stream != 0 && stream != 1))
        return fail(nullptr, MOCHII_ERR_BAD_PARAM, "mochii_philox_uniforms: bad argument");
    if (n == 0) return MOCHII_OK;
    double* d = nullptr;
    cudaError_t e = cudaMalloc(&d, (size_t)n * 8);
    if (e == cudaSuccess) e = launch_philox((uint64_t)seed, (uint32_t)stream, (uint64_t)packet, n0, n, d);
    if (e == cudaSuccess) e = cudaMemcpy(out, d, (size_t)n * 8, cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (e != cudaSuccess) return fail(nullptr, MOCHII_ERR_CUDA, std::string("mochii_philox_uniforms: ") + cudaGetErrorString(e));
    return MOCHII_OK;
}

extern "C" int mochii_walk_leaves(mochii_ctx* c, int64_t nray, const double* rays, int max_steps, int32_t* leaves,
                                  int32_t* nsteps) {
    if (!c || !rays || !leaves || !nsteps || nray < 0 || max_steps < 1) return MOCHII_ERR_BAD_PARAM;
    if (nray == 0) return MOCHII_OK;
    double* dr = nullptr;
    int *dl = nullptr, *dn = nullptr;
    CK(c, cudaMallocAsync(&dr, nray * 6 * 8, c->stream));
    CK(c, cudaMallocAsync(&dl, (size_t)nray * max_steps * 4, c->stream));
    CK(c, cudaMallocAsync(&dn, nray * 4, c->stream));
    CK(c, cudaMemcpyAsync(dr, rays, nray * 6 * 8, cudaMemcpyHostToDevice, c->stream));
    CK(c, launch_walk(c, dr, nray, max_steps, dl, dn));
    CK(c, cudaMemcpyAsync(leaves, dl, (size_t)nray * max_steps * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaMemcpyAsync(nsteps, dn, nray * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaFreeAsync(dr, c->stream));
    CK(c, cudaFreeAsync(dl, c->stream));
    CK(c, cudaFreeAsync(dn, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return MOCHII_OK;
}

extern "C" int mochii_launch_records(mochii_ctx* c, int64_t ip0, int64_t n, double* out8) {
    if (!c || !out8 || n < 0 || ip0 < 0) return MOCHII_ERR_BAD_PARAM;
    if (n == 0) return MOCHII_OK;
    double* d = nullptr;
    CK(c, cudaMallocAsync(&d, n * 8 * 8, c->stream));
    CK(c, launch_records(c, ip0, n, d));
    CK(c, cudaMemcpyAsync(out8, d, n * 8 * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaFreeAsync(d, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return MOCHII_OK;
}

// Launch records staged in the library's static device array (see
// transport.cu): no device allocation; n <= 65536 per call.
extern "C" int mochii_launch_records_noalloc(mochii_ctx* c, int64_t ip0, int64_t n, double* out8) {
    if (!c || !out8 || n < 0 || ip0 < 0) return fail(c, MOCHII_ERR_BAD_PARAM, "mochii_launch_records_noalloc: bad argument");
    if (n > noalloc_max_records())
        return fail(c, MOCHII_ERR_BAD_PARAM,
                    "mochii_launch_records_noalloc: n exceeds the 65536 records of the static staging array");
    if (n == 0) return MOCHII_OK;
    // the static array's address is per device: take it on the context's own
    // device, never on whichever device the caller left current
    int dev = -1;
    CK(c, cudaGetDevice(&dev));
    if (dev != c->device)
        return fail(c, MOCHII_ERR_BAD_PARAM,
                    "mochii_launch_records_noalloc: the current device is not the context's device; "
                    "call cudaSetDevice on the context's device first");
    CK(c, launch_records_noalloc(c, ip0, n, out8));
    return MOCHII_OK;
}

// Diffuse launch records (x, y, z, kx, ky, kz, E, inu) of packets ip0..ip0+n-1
// from the current state: diffuse_build + gen_diffuse_photon_qmc.
extern "C" int mochii_diffuse_records(mochii_ctx* c, int64_t ip0, int64_t n, double* out8, double* lum,
                                      int64_t* nphot) {
    if (!c || n < 0 || ip0 < 0) return MOCHII_ERR_BAD_PARAM;
    if (!c->par.diffuse_field) return fail(c, MOCHII_ERR_BAD_PARAM, "par%diffuse_field is off");
    double total = 0.0;
    CK(c, diffuse_build(c, &total));
    if (lum) *lum = total;
    if (nphot) *nphot = total > 0.0 ? std::llround(total / (c->band.ion_Ltot / (double)c->par.nphotons)) : 0;
    if (n == 0 || total <= 0.0) return MOCHII_OK;
    if (n > c->rec.cap) return fail(c, MOCHII_ERR_BAD_PARAM, "n exceeds the record buffer");
    CK(c, launch_diffuse_chunk(c, total, ip0, n));
    CK(c, launch_records_from_buffer(c, n, out8));
    return MOCHII_OK;
}
