// Diffuse ground-recombination packets on the device (diffuse_mod.f90 with
// the Milne ground-continuum spectra of milne_recomb_spectrum_mod.f90).
//
// Per pass: k_diffuse_lum evaluates, per leaf, the luminosity of the three
// ground channels (H II -> H I 1s, He II -> He I 1^1S, He III -> He II 1s):
// L = n_e n_ion (alpha_A - alpha_B)(T) <E>_Milne(T) V  (diffuse_mod.f90:78-90);
// a device prefix sum over leaves turns the leaf totals into the emission
// CDF; the packet count is nint(L_diffuse / L_packet) (:116).  k_launch_diffuse
// then draws leaf (binary search of the CDF), position in the leaf, isotropic
// direction, channel and Milne energy from the 9-dimensional diffuse Sobol
// stream (diffuse_mod.f90:221-296) and writes the same packet records as the
// stellar launch, so the walk kernel is shared.  With par%hei_diffuse a
// fourth channel carries the He I excited-level recombination radiation
// (diffuse_mod.f90:96-106, 274-284): the 2^3S and 584 A lines and the 2^1S
// two-photon continuum above the H I edge.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>

#include "ctx.h"
#include "diffuse.h"
#include "metals.cuh"
#include "physics.cuh"
#include "qmc.cuh"
#include "records.cuh"
#include "transport.h"

namespace mochii {

// ---- host: Milne tables (milne_recomb_spectrum_mod.f90:99-228) -------------
// Quadratically clustered x = (E - E_th)/kT nodes on [0, 60] (512), log T
// nodes 1e2-1e6 K (192); per (T, channel) the energy-luminosity CDF of the
// photon PDF E^2 sigma(E) exp(-x) by Simpson panels truncated at eion_max,
// the mean x under the number PDF and the in-band photon fraction.
void milne_tables_build(double eion_max, MilneHost& m) {
    const double XMAX = 60.0;
    const double eth[3] = {kEthHI, kEthHeI, kEthHeII};
    m.xg.resize(kMilneNX);
    m.lgT.resize(kMilneNT);
    for (int ix = 0; ix < kMilneNX; ++ix) {
        const double t = (double)ix / (double)(kMilneNX - 1);
        m.xg[ix] = XMAX * t * t;
    }
    for (int it = 0; it < kMilneNT; ++it)
        m.lgT[it] = std::log10(1.0e2) + (std::log10(1.0e6) - std::log10(1.0e2)) * (double)it / (double)(kMilneNT - 1);
    m.cdf.assign((size_t)3 * kMilneNT * kMilneNX, 0.0);
    m.xbar.assign((size_t)3 * kMilneNT, 0.0);
    m.frac.assign((size_t)3 * kMilneNT, 0.0);
    for (int ich = 0; ich < 3; ++ich) {
        for (int it = 0; it < kMilneNT; ++it) {
            double* c = &m.cdf[((size_t)ich * kMilneNT + it) * kMilneNX];
            const double kT = kKboltz * std::pow(10.0, m.lgT[it]) / kEv2erg;
            auto shape = [&](double x) {
                const double E = eth[ich] + x * kT;
                const double s = ich == 0 ? sigma_HI(E) : ich == 1 ? sigma_HeI(E) : sigma_HeII(E);
                return E * E * s * std::exp(-x);
            };
            const double x_hi = std::min(XMAX, (eion_max - eth[ich]) / kT);
            if (x_hi <= 0.0) {
                std::fill(c, c + kMilneNX, 1.0);
                continue;
            }
            double sn = 0.0, se = 0.0, sxn = 0.0;
            c[0] = 0.0;
            for (int ix = 1; ix < kMilneNX; ++ix) {
                const double xa = m.xg[ix - 1], xb = std::min(m.xg[ix], x_hi);
                if (xb > xa) {
                    const double xm = 0.5 * (xa + xb);
                    const double fa = shape(xa), fm = shape(xm), fb = shape(xb);
                    sn = sn + (xb - xa) / 6.0 * (fa + 4.0 * fm + fb);
                    se = se + (xb - xa) / 6.0 *
                                  (fa * (eth[ich] + xa * kT) + 4.0 * fm * (eth[ich] + xm * kT) + fb * (eth[ich] + xb * kT));
                    sxn = sxn + (xb - xa) / 6.0 * (fa * xa + 4.0 * fm * xm + fb * xb);
                }
                c[ix] = se;
            }
            double tail = sn;
            for (double xa = x_hi; xa < XMAX;) {
                const double xb = std::min(xa + 0.25, XMAX), xm = 0.5 * (xa + xb);
                tail = tail + (xb - xa) / 6.0 * (shape(xa) + 4.0 * shape(xm) + shape(xb));
                xa = xb;
            }
            if (se > 0.0) {
                for (int ix = 0; ix < kMilneNX; ++ix) c[ix] = c[ix] / se;
            } else {
                std::fill(c, c + kMilneNX, 1.0);
            }
            c[kMilneNX - 1] = 1.0;
            m.xbar[(size_t)ich * kMilneNT + it] = sxn / std::max(sn, kTinest);
            m.frac[(size_t)ich * kMilneNT + it] = sn / std::max(tail, kTinest);
        }
    }
}

// ---- host: He I two-photon table (hei_twophoton_mod.f90:97-192) ------------
// A(y) linearly interpolated between the tabulated points; its integral over
// [0, 1] by Simpson panels per table interval (midpoints interpolated) is the
// normalisation; on the in-band window [13.598, min(20.62, eion_max)] / 20.62
// 1023 equal Simpson panels give the photons and energy per decay (two
// photons per decay) and the CDF of the energy density y A(y).
bool hei_2ph_build(const std::string& path, double eion_max, HeI2phHost& h) {
    std::vector<double> ty, ta;
    if (FILE* f = std::fopen(path.c_str(), "r")) {
        double y, a;
        while (std::fscanf(f, "%lf %lf", &y, &a) == 2) {
            ty.push_back(y);
            ta.push_back(a);
        }
        std::fclose(f);
    }
    const int n = (int)ty.size();
    if (n < 4) return false;
    auto shape = [&](double y) {
        if (y <= ty[0] || y >= ty[n - 1]) return 0.0;
        int i = 0;
        while (i < n - 2 && ty[i + 1] < y) ++i;
        return ta[i] + (ta[i + 1] - ta[i]) * (y - ty[i]) / (ty[i + 1] - ty[i]);
    };
    double tot = 0.0;
    for (int i = 0; i < n - 1; ++i) {
        const double ya = ty[i], yb = ty[i + 1];
        tot = tot + (yb - ya) / 6.0 * (ta[i] + 4.0 * shape(0.5 * (ya + yb)) + ta[i + 1]);
    }
    if (tot <= 0.0) return false;
    h.cdf_e.assign(kHe2phN, 1.0);
    h.grid_y.assign(kHe2phN, 0.0);
    const double y_lo = kEthHI / kHe2phEtot, y_hi = std::min(kHe2phEtot, eion_max) / kHe2phEtot;
    if (y_hi <= y_lo) {
        h.n_per_decay = h.e_per_decay = 0.0;
        for (double& g : h.grid_y) g = y_lo;
        return true;
    }
    double an = 0.0, ae = 0.0, seg = 0.0;
    h.grid_y[0] = y_lo;
    h.cdf_e[0] = 0.0;
    for (int i = 1; i < kHe2phN; ++i) {
        const double ya = y_lo + (y_hi - y_lo) * (double)(i - 1) / (double)(kHe2phN - 1);
        const double yb = y_lo + (y_hi - y_lo) * (double)i / (double)(kHe2phN - 1);
        const double ym = 0.5 * (ya + yb);
        const double fa = shape(ya), fm = shape(ym), fb = shape(yb);
        const double w = (fa * ya + 4.0 * fm * ym + fb * yb);
        an = an + (yb - ya) / 6.0 * (fa + 4.0 * fm + fb);
        ae = ae + (yb - ya) / 6.0 * w * kHe2phEtot;
        seg = seg + (yb - ya) / 6.0 * w;
        h.grid_y[i] = yb;
        h.cdf_e[i] = seg;
    }
    h.n_per_decay = 2.0 * an / tot;
    h.e_per_decay = 2.0 * ae / tot;
    for (double& c : h.cdf_e) c = seg > 0.0 ? c / seg : 1.0;
    h.cdf_e[kHe2phN - 1] = 1.0;
    return true;
}

namespace {

constexpr int kThreads = 256;

// hei_branch_energies (diffuse_mod.f90:308-325 with hei_cascade_mod.f90): the
// in-band energy per case-B He II recombination through the 2^3S line
// (19.82 eV), the 584 A line when its trapped photon ionizes hydrogen
// (21.22 eV; escape closure p = 1 / (1 + 77 x(He0) / (sqrt(T) x(H0)))), and
// the two-photon continuum of 2^1S and of the 2^1P decays converted to it.
// Branch fractions from the Benjamin, Skillman & Smits (1999) effective
// coefficients normalised by their sum, T clamped to [3e3, 2e4] K.
__device__ __forceinline__ void hei_branches(const HeI2phDev& h, double T, double xHI, double xHeI, double& e3s,
                                             double& e1p, double& e1s) {
    const double Tc = fmin(fmax(T, 3.0e3), 2.0e4) / 1.0e4;
    const double a3 = 2.10e-13 * pow(Tc, -0.381);
    const double a1s = 2.06e-14 * pow(Tc, -0.451);
    const double a1p = 4.17e-14 * pow(Tc, -0.695);
    const double sum = a3 + a1s + a1p;
    const double f3s = a3 / sum, f1s = a1s / sum, f1p = a1p / sum;
    const double p584 = 1.0 / (1.0 + 77.0 / sqrt(fmax(T, kTinest)) * fmax(xHeI, 0.0) / fmax(xHI, kTinest));
    e3s = f3s * 19.82;
    e1p = f1p * p584 * 21.22;
    e1s = (f1s + f1p * (1.0 - p584)) * h.e_per_decay;
}

// hei_2ph_sample_energy (hei_twophoton_mod.f90:199-219): bisection of the
// energy CDF and linear interpolation within the bracket.
__device__ double hei_2ph_sample(const HeI2phDev& h, double u) {
    const double uu = fmin(fmax(u, 0.0), 1.0);
    int lo = 0, hi = kHe2phN - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi + 2) / 2 - 1;
        if (uu > h.cdf_e[mid]) lo = mid; else hi = mid;
    }
    const double cl = h.cdf_e[lo], ch = h.cdf_e[hi];
    const double y = ch > cl ? h.grid_y[lo] + (h.grid_y[hi] - h.grid_y[lo]) * (uu - cl) / (ch - cl) : h.grid_y[lo];
    return y * kHe2phEtot;
}

struct DiffArgs {
    const double* nH;
    const double* xHI;
    const double* xHeI;
    const double* xHeII;
    const double* ne;
    const double* Te;
    double* ch;        // 4 x nleaf (channel luminosities, leaf-major)
    double* tot;       // nleaf leaf totals, then their inclusive prefix sum
    MilneDev m;
    HeI2phDev he;
    const double4* lg;   // octree leaf geometry (per-leaf volume), null on the Cartesian grid
    long long nleaf;
    double yHe, vol, d2cm, eion_max;
    RateSel rs;
    int energy_model;  // 0 milne, 1 exponential, 2 threshold
    int hei;           // the He I excited channel (par%hei_diffuse)
};

// milne_tbracket (:286-297): it is 1-based as in the reference.
__device__ __forceinline__ void tbracket(const MilneDev& m, double T, int& it, double& w) {
    double s = (log10(fmax(T, kTinest)) - m.lgT0) / m.dlgT;
    s = fmin(fmax(s, 0.0), (double)(kMilneNT - 1));
    it = min((int)s + 1, kMilneNT - 1);
    w = s - (double)(it - 1);
}

// milne_energy_per_recomb (:302-312).
__device__ double energy_per_recomb(const MilneDev& m, int ich, double T, double eth) {
    int it;
    double w;
    tbracket(m, T, it, w);
    const double xb = (1.0 - w) * m.xbar[ich * kMilneNT + it - 1] + w * m.xbar[ich * kMilneNT + it];
    const double fk = (1.0 - w) * m.frac[ich * kMilneNT + it - 1] + w * m.frac[ich * kMilneNT + it];
    return fk * (eth + xb * (kKboltz * T / kEv2erg));
}

// milne_sample_energy (:320-350): binary search of the log-T-interpolated CDF,
// then linear inversion inside the bracket.
__device__ double milne_sample(const MilneDev& m, int ich, double T, double u, double eth, double eion_max) {
    int it;
    double w;
    tbracket(m, T, it, w);
    const double kT = kKboltz * T / kEv2erg;
    const double uu = fmin(fmax(u, 0.0), 1.0);
    const double* c0 = m.cdf + ((size_t)ich * kMilneNT + it - 1) * kMilneNX;
    const double* c1 = c0 + kMilneNX;
    int lo = 1, hi = kMilneNX;
    double ca = (1.0 - w) * c0[0] + w * c1[0];
    double cb = (1.0 - w) * c0[kMilneNX - 1] + w * c1[kMilneNX - 1];
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        const double cm = (1.0 - w) * c0[mid - 1] + w * c1[mid - 1];
        if (uu > cm) { lo = mid; ca = cm; } else { hi = mid; cb = cm; }
    }
    const double x = cb > ca ? m.xg[lo - 1] + (m.xg[hi - 1] - m.xg[lo - 1]) * (uu - ca) / (cb - ca) : m.xg[lo - 1];
    return fmin(eth + x * kT, eion_max * (1.0 - 1.0e-12));
}

__global__ void k_diffuse_lum(const DiffArgs a) {
    for (long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x; il < a.nleaf;
         il += (long long)gridDim.x * blockDim.x) {
        double c0 = 0.0, c1 = 0.0, c2 = 0.0, c3 = 0.0;
        const double nH = a.nH[il];
        if (nH > 0.0) {
            const double T = a.Te[il], ne = a.ne[il];
            const double kT = kKboltz * T / kEv2erg;
            const double xHeIII = fmax(0.0, 1.0 - a.xHeI[il] - a.xHeII[il]);
            const double nHII = nH * (1.0 - a.xHI[il]);
            const double nHeII = nH * a.yHe * a.xHeII[il];
            const double nHeIII = nH * a.yHe * xHeIII;
            double e0, e1, e2;
            if (a.energy_model == 0) {
                e0 = energy_per_recomb(a.m, 0, T, kEthHI);
                e1 = energy_per_recomb(a.m, 1, T, kEthHeI);
                e2 = energy_per_recomb(a.m, 2, T, kEthHeII);
            } else if (a.energy_model == 1) {
                e0 = kEthHI + kT; e1 = kEthHeI + kT; e2 = kEthHeII + kT;
            } else {
                e0 = kEthHI; e1 = kEthHeI; e2 = kEthHeII;
            }
            double vol = a.vol;
            if (a.lg) {
                const double w = 2.0 * a.lg[il].w * a.d2cm;
                vol = w * w * w;
            }
            c0 = ne * nHII * (alphaA_HII(a.rs, T) - alphaB_HII(a.rs, T)) * e0 * kEv2erg * vol;
            c1 = ne * nHeII * (alphaA_HeII(a.rs, T) - alphaB_HeII(a.rs, T)) * e1 * kEv2erg * vol;
            c2 = ne * nHeIII * (alphaA_HeIII(a.rs, T) - alphaB_HeIII(a.rs, T)) * e2 * kEv2erg * vol;
            if (a.hei) {   // channel 4: every case-B He II recombination through the n = 2 cascade
                double e3s, e1p, e1s;
                hei_branches(a.he, T, a.xHI[il], a.xHeI[il], e3s, e1p, e1s);
                c3 = ne * nHeII * alphaB_HeII(a.rs, T) * vol * kEv2erg * ((e3s + e1p) + e1s);
            }
        }
        a.ch[4 * il + 0] = c0;
        a.ch[4 * il + 1] = c1;
        a.ch[4 * il + 2] = c2;
        a.ch[4 * il + 3] = c3;
        a.tot[il] = ((c0 + c1) + c2) + c3;
    }
}

struct DiffLaunchArgs {
    const QmcTables* qmc;
    const double* cum;     // inclusive prefix sum of the leaf totals
    const double* ch;
    const double* Te;
    const double* xHI;
    const double* xHeI;
    const double* eedge;
    MilneDev m;
    HeI2phDev he;
    MetalDev metal;
    const double4* lg;   // octree leaf geometry, null on the Cartesian grid
    DustDev dust;        // grain optics; dust.n == 0 without
    int xs, scatter;     // grain / FUV record terms; scattered flights
    double eion_min;
    double total, org[3], dcell, eion_max;
    int n[3], nnu, nfuv, energy_model;
    long long nleaf;
};

// The emitting leaf of gen_diffuse_photon_qmc: the first leaf whose
// normalised CDF reaches u1.
__device__ __forceinline__ long long diffuse_leaf(const DiffLaunchArgs& a, double u0) {
    long long lo = 1, hi = a.nleaf;
    while (lo < hi) {
        const long long mid = (lo + hi) / 2;
        if (a.cum[mid - 1] / a.total < u0) lo = mid + 1; else hi = mid;
    }
    return lo - 1;
}

// gen_diffuse_photon_qmc (diffuse_mod.f90:221-296) and dda_init.  With
// rec.order (packet_order 'coherent') record i holds chunk packet order[i].
template <typename R>
__global__ void __launch_bounds__(kThreads) k_launch_diffuse(const DiffLaunchArgs a, PacketRecords rec, long long ip0,
                                                             long long n) {
    __shared__ QmcTables sq;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(a.qmc);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&sq);
        for (int i = threadIdx.x; i < (int)(sizeof(QmcTables) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t ip = (uint64_t)(ip0 + (rec.order ? (long long)rec.order[i] : i));
    double u[9];
#pragma unroll
    for (int d = 0; d < 9; ++d) u[d] = qmc_uniform(sq, ip, d, 1);
    const long long il = diffuse_leaf(a, u[0]);
    double pos[3];
    if (a.lg) {   // leaf centre and half width of the octree leaf
        const double4 g = a.lg[il];
        pos[0] = g.x + (2.0 * u[1] - 1.0) * g.w;
        pos[1] = g.y + (2.0 * u[2] - 1.0) * g.w;
        pos[2] = g.z + (2.0 * u[3] - 1.0) * g.w;
    } else {
        const int ix = (int)(il % a.n[0]), iy = (int)((il / a.n[0]) % a.n[1]);
        const int iz = (int)(il / ((long long)a.n[0] * a.n[1]));
        const double half = 0.5 * a.dcell;
        pos[0] = (a.org[0] + ((double)ix + 0.5) * a.dcell) + (2.0 * u[1] - 1.0) * half;
        pos[1] = (a.org[1] + ((double)iy + 0.5) * a.dcell) + (2.0 * u[2] - 1.0) * half;
        pos[2] = (a.org[2] + ((double)iz + 0.5) * a.dcell) + (2.0 * u[3] - 1.0) * half;
    }
    const double cost = 2.0 * u[4] - 1.0;
    const double sint = sqrt(1.0 - cost * cost);
    double sphi, cphi;
    sincos(kTwoPi * u[5], &sphi, &cphi);
    const double kk[3] = {sint * cphi, sint * sphi, cost};
    const double w0 = a.ch[4 * il], w1 = a.ch[4 * il + 1], w2 = a.ch[4 * il + 2], w3 = a.ch[4 * il + 3];
    const double uu = u[6] * (((w0 + w1) + w2) + w3);
    int ch;
    double eph;
    if (uu <= w0) { ch = 0; eph = kEthHI; }
    else if (uu <= w0 + w1) { ch = 1; eph = kEthHeI; }
    else if (uu <= w0 + w1 + w2) { ch = 2; eph = kEthHeII; }
    else { ch = 3; eph = kEthHI; }
    if (ch <= 2) {
        const double T = a.Te[il];
        if (a.energy_model == 0) eph = milne_sample(a.m, ch, T, u[7], eph, a.eion_max);
        else if (a.energy_model == 1) eph = eph + (kKboltz * T / kEv2erg) * (-log(fmax(u[7], kTinest)));
        eph = fmin(eph, a.eion_max * 0.999);
    } else {   // the He I excited channel: 2^3S line, 584 A line or two-photon continuum
        double e3s, e1p, e1s;
        hei_branches(a.he, a.Te[il], a.xHI[il], a.xHeI[il], e3s, e1p, e1s);
        const double ub = u[7] * ((e3s + e1p) + e1s);
        if (ub <= e3s) eph = 19.82;
        else if (ub <= e3s + e1p) eph = 21.22;
        else eph = hei_2ph_sample(a.he, u[8]);
    }
    // ion_bin_of without the FUV bins (ion_band_mod.f90:624-646)
    int blo = 1, bhi = a.nnu;
    while (blo < bhi) {
        const int mid = (blo + bhi + 1) / 2;
        if (a.eedge[mid - 1] <= eph) blo = mid; else bhi = mid - 1;
    }
    const int inu = min(max(blo, a.nfuv + 1), a.nnu) - 1;
    if (a.lg) write_record_amr<R>(rec, i, pos, kk, eph, inu, (int)il);
    else write_record<R>(rec, i, pos, kk, eph, inu, a.org, a.dcell, a.n);
    if (a.xs) write_grain_record<R>(rec, i, a.dust, a.scatter, a.eion_min, eph, pos, kk, a.lg ? 0 : 1);
    if (a.metal.ntr > 0) write_metal_record<R>(rec, a.metal, i, eph);
}

// Walk-order keys of packet_order 'coherent' for the diffuse packets
// ip0 .. ip0+n-1 on the Cartesian grid: the emitting leaf and the direction
// uniforms of gen_diffuse_photon_qmc reduced to diffuse_coherent_key.
__global__ void __launch_bounds__(kThreads) k_diffuse_keys(const DiffLaunchArgs a, long long ip0, long long n,
                                                           unsigned* __restrict__ key) {
    __shared__ QmcTables sq;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(a.qmc);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&sq);
        for (int i = threadIdx.x; i < (int)(sizeof(QmcTables) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t ip = (uint64_t)(ip0 + i);
    const long long il = diffuse_leaf(a, qmc_uniform(sq, ip, 0, 1));
    const int ix = (int)(il % a.n[0]), iy = (int)((il / a.n[0]) % a.n[1]);
    const int iz = (int)(il / ((long long)a.n[0] * a.n[1]));
    key[i] = diffuse_coherent_key(qmc_uniform(sq, ip, 4, 1), qmc_uniform(sq, ip, 5, 1), ix, iy, iz, a.n);
}

int nblk(long long work, int threads, int cap) {
    long long b = (work + threads - 1) / threads;
    return (int)(b < 1 ? 1 : b > cap ? cap : b);
}

}  // namespace

// Per-leaf diffuse luminosities and their prefix sum; returns the total
// diffuse luminosity (one 8-byte device-to-host read).
cudaError_t diffuse_build(mochii_ctx* c, double* total) {
    DiffArgs a;
    a.nH = c->nH; a.xHI = c->xHI; a.xHeI = c->xHeI; a.xHeII = c->xHeII; a.ne = c->ne; a.Te = c->Te;
    a.ch = c->dif.ch;
    a.tot = c->dif.tot;
    a.m = c->dif.m;
    a.nleaf = c->grid.nleaf;
    a.yHe = c->par.He_abund;
    const double w = c->grid.dcell * c->par.distance2cm;
    a.vol = w * w * w;
    a.lg = c->oct.ncells > 0 ? c->oct.lgeo : nullptr;
    a.d2cm = c->par.distance2cm;
    a.eion_max = c->par.eion_max;
    a.rs.hui_gnedin = c->par.recomb_hui_gnedin;
    a.rs.dere_hybrid = c->par.ci_dere_hybrid;
    a.energy_model = c->par.diffuse_model;
    a.he = c->dif.he;
    a.hei = c->par.hei_diffuse ? 1 : 0;
    k_diffuse_lum<<<nblk(a.nleaf, kThreads, 148 * 16), kThreads, 0, c->stream>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t tmp = c->dif.scan_bytes;
    e = cub::DeviceScan::InclusiveSum(c->dif.scan_tmp, tmp, c->dif.tot, c->dif.tot, (int)a.nleaf, c->stream);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(total, c->dif.tot + (a.nleaf - 1), sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(c->stream);
}

size_t diffuse_scan_bytes(long long nleaf) {
    size_t bytes = 0;
    cub::DeviceScan::InclusiveSum(nullptr, bytes, (double*)nullptr, (double*)nullptr, (int)nleaf);
    return bytes;
}

namespace {
DiffLaunchArgs diffuse_launch_args(mochii_ctx* c, double total) {
    DiffLaunchArgs a;
    a.qmc = c->tab.qmc;
    a.cum = c->dif.tot;
    a.ch = c->dif.ch;
    a.Te = c->Te;
    a.xHI = c->xHI;
    a.xHeI = c->xHeI;
    a.eedge = c->tab.eedge;
    a.m = c->dif.m;
    a.he = c->dif.he;
    a.total = total;
    a.org[0] = c->grid.xmin; a.org[1] = c->grid.ymin; a.org[2] = c->grid.zmin;
    a.metal = c->metal;
    a.lg = c->oct.ncells > 0 ? c->oct.lgeo : nullptr;
    a.dust = c->dust;
    a.xs = c->xscore ? 1 : 0;
    a.scatter = c->scatter ? 1 : 0;
    a.eion_min = c->par.eion_min;
    a.dcell = c->grid.dcell;
    a.eion_max = c->par.eion_max;
    a.n[0] = c->grid.nx; a.n[1] = c->grid.ny; a.n[2] = c->grid.nz;
    a.nnu = c->nnu;
    a.nfuv = c->band.nfuv_band;
    a.energy_model = c->par.diffuse_model;
    a.nleaf = c->grid.nleaf;
    return a;
}
}  // namespace

cudaError_t launch_diffuse_keys(mochii_ctx* c, double total, long long ip0, long long n, unsigned* key) {
    const DiffLaunchArgs a = diffuse_launch_args(c, total);
    k_diffuse_keys<<<nblk(n, kThreads, 1 << 30), kThreads, 0, c->stream>>>(a, ip0, n, key);
    return cudaGetLastError();
}

cudaError_t launch_diffuse_chunk(mochii_ctx* c, double total, long long ip0, long long n, const int* order) {
    const DiffLaunchArgs a = diffuse_launch_args(c, total);
    PacketRecords r = packet_records(c);
    r.order = order;
    if (c->fp32) k_launch_diffuse<float><<<nblk(n, kThreads, 1 << 30), kThreads, 0, c->stream>>>(a, r, ip0, n);
    else k_launch_diffuse<double><<<nblk(n, kThreads, 1 << 30), kThreads, 0, c->stream>>>(a, r, ip0, n);
    return cudaGetLastError();
}

}  // namespace mochii
