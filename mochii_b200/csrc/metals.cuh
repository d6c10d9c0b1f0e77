// Device side of the trace-metal registry (species_mod.f90): packet cross
// sections, rate coefficients, the per-(leaf, T) rate cache, the cascade
// sums that feed hydrogen's balance and the n_e closure, the charge-exchange
// hydrogen root (ion_balance_mod.f90:177-208), the n_e closure of the written
// state (:235-253), the stage fractions behind the packet opacity, and the
// metal cooling / heating terms of the thermal balance (thermal_mod.f90:53-71).
// All FP64; element order j, threshold order k (species.h).
#pragma once
#include "physics.cuh"
#include "records.cuh"
#include "species.h"

namespace mochii {

// sigma_vy95, photo_xsec.f90:69-82 (Verner & Yakovlev 1995 outer shell).
MHD double sigma_vy95(double E, double Eth, double E0, double s0, double ya, double P, double yw, double l) {
    if (E < Eth) return 0.0;
    const double y = E / E0;
    const double Q = 5.5 + l - 0.5 * P;
    const double ym1 = y - 1.0;
    return s0 * ((ym1 * ym1 + yw * yw) * pow(y, -Q) * pow(1.0 + sqrt(y / ya), -P)) * 1.0e-18;
}

// species_sigma (species_mod.f90:763-778), threshold order k.
__device__ __forceinline__ double metal_sigma(const MetalDev& m, int k, double E) {
    const double* c = m.photo + 8 * k;
    if (m.form[k] == 2) return sigma_vy95(E, c[0], c[1], c[2], c[3], c[4], c[5], c[6]);
    return sigma_vfky96(E, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7]);
}

// Number of active transitions (E >= E_th) of a packet: the prefix that
// species_packet_cross_sections (species_mod.f90:263-275) fills.
__device__ __forceinline__ int metal_nactive(const MetalDev& m, double E) {
    int n = 0;
    while (n < m.ntr && !(E < __ldg(m.eth + n))) ++n;
    return n;
}

// Metal part of a packet record: E and sigma_k * 1e18 for the active prefix.
template <typename R>
__device__ __forceinline__ void write_metal_record(const PacketRecords& rec, const MetalDev& m, long long i, double E) {
    rec.E[i] = E;
    R* ms = static_cast<R*>(rec.msig);
    const int nm = metal_nactive(m, E);
    for (int k = 0; k < nm; ++k) ms[k * rec.cap + i] = (R)(metal_sigma(m, k, E) * 1.0e18);
}

// alpha_rec (species_mod.f90:428-447): Badnell RR (or the RR2 power law) plus
// Badnell DR and the Shull & Van Steenberg DR2 term.
static __device__ __noinline__ double metal_alpha_rec(const MetalTr& r, double T) {
    double a;
    if (r.has_rr2) {
        a = r.rr2[0] * pow(T / 1.0e4, -r.rr2[1]);
    } else {
        const double s0 = sqrt(T / r.rr[2]), s1 = sqrt(T / r.rr[3]);
        const double b = r.rr[1] + r.rr[4] * exp(-r.rr[5] / T);
        a = r.rr[0] / (s0 * pow(1.0 + s0, 1.0 - b) * pow(1.0 + s1, 1.0 + b));
    }
    if (r.ndr > 0 || r.has_dr2) {
        const double t15 = pow(T, -1.5);
        for (int k = 0; k < r.ndr; ++k) a = a + t15 * r.dr_c[k] * exp(-r.dr_e[k] / T);
        if (r.has_dr2) a = a + r.dr2[0] * t15 * exp(-r.dr2[2] / T) * (1.0 + r.dr2[1] * exp(-r.dr2[3] / T));
    }
    return a;
}

// cx_rate (species_mod.f90:452-487): the seven charge-exchange fit forms.
static __device__ __noinline__ double metal_cx_rate(int form, const double* c, double T) {
    double t4 = T / 1.0e4, k, lnT;
    switch (form) {
        case 1:
            k = c[0] * pow(T / 300.0, c[1]);
            if (c[2] != 0.0) k = k * exp(-c[2] / t4);
            return k;
        case 2: return c[0] * pow(t4, c[1]) + c[2] * pow(t4, c[3]);
        case 3: return (c[0] * pow(t4, c[1]) + c[2] * pow(t4, c[3])) * exp(-c[4] / T);
        case 4:
            lnT = log(T);
            return exp(c[0] + lnT * (c[1] + lnT * (c[2] + lnT * (c[3] + lnT * c[4]))));
        case 5:
            lnT = log(T);
            return exp(c[0] + lnT * (c[1] + lnT * (c[2] + lnT * (c[3] + lnT * c[4]))) - c[5] / t4);
        case 6:
            t4 = fmin(fmax(t4, 0.5), 5.0);
            k = c[0] * pow(t4, c[1]) * (1.0 + c[2] * exp(c[3] * t4));
            return fmax(k, 0.0);
        case 7:
            t4 = fmin(fmax(t4, 0.5), 5.0);
            k = c[0] * pow(t4, c[1]) * (1.0 + c[2] * exp(c[3] * t4)) * exp(-c[4] / t4);
            return fmax(k, 0.0);
        default: return 0.0;
    }
}

// The (leaf, T) rate cache of species_ne_prepare (species_mod.f90:517-536).
struct MetalCache {
    double gam[kMaxTr], ci[kMaxTr], rec[kMaxTr], cxi[kMaxTr], cxr[kMaxTr];
};

// The four T-dependent coefficients of transition j at T: collisional
// ionisation, recombination, CX ionisation, CX recombination.
__device__ __forceinline__ double metal_coef(const MetalTr& r, int c, double T) {
    switch (c) {
        case 0: return voronov(T, r.ci[0], r.ci[1], r.ci[2], r.ci[3], r.ci[4]) * r.cidr;
        case 1: return metal_alpha_rec(r, T);
        case 2: return r.cxi_form > 0 ? metal_cx_rate(r.cxi_form, r.cxi, T) : 0.0;
        default: return r.cxr_form > 0 ? metal_cx_rate(r.cxr_form, r.cxr, T) : 0.0;
    }
}

// species_ne_prepare (species_mod.f90:517-536).  Inside the range of the T
// table the coefficients come from 4-point Lagrange interpolation of their
// logarithms in ln T (relative error ~1e-12 on the 4096-node table of the
// thermal solve); the charge-exchange fits clamped in T (forms 6, 7) and
// every T outside the table are evaluated directly.
static __device__ __noinline__ void metal_prepare(const MetalDev& m, long long il, double T, MetalCache& c) {
    int i0 = -1;
    double w0 = 0.0, w1 = 0.0, w2 = 0.0, w3 = 0.0;
    if (m.tnt > 0) {
        const double s = (log(T) - m.tu0) / m.tdu;
        const int i = (int)floor(s);
        if (i >= 1 && i <= m.tnt - 3) {
            const double t = s - (double)i;
            w0 = -t * (t - 1.0) * (t - 2.0) / 6.0;
            w1 = (t + 1.0) * (t - 1.0) * (t - 2.0) / 2.0;
            w2 = -(t + 1.0) * t * (t - 2.0) / 2.0;
            w3 = (t + 1.0) * t * (t - 1.0) / 6.0;
            i0 = i - 1;
        }
    }
    for (int j = 0; j < m.ntr; ++j) {
        const MetalTr& r = m.tr[j];
        c.gam[j] = m.egam[il * m.ntr + j];
        if (i0 >= 0) {
            const double* L = m.ttab + (size_t)j * 4 * m.tnt + i0;
            c.ci[j] = exp(w0 * L[0] + w1 * L[1] + w2 * L[2] + w3 * L[3]);
            L += m.tnt;
            c.rec[j] = exp(w0 * L[0] + w1 * L[1] + w2 * L[2] + w3 * L[3]);
            L += m.tnt;
            c.cxi[j] = r.cxi_form <= 0 ? 0.0 : r.cxi_form >= 6 ? metal_cx_rate(r.cxi_form, r.cxi, T)
                                                             : exp(w0 * L[0] + w1 * L[1] + w2 * L[2] + w3 * L[3]);
            L += m.tnt;
            c.cxr[j] = r.cxr_form <= 0 ? 0.0 : r.cxr_form >= 6 ? metal_cx_rate(r.cxr_form, r.cxr, T)
                                                             : exp(w0 * L[0] + w1 * L[1] + w2 * L[2] + w3 * L[3]);
        } else {
            c.ci[j] = metal_coef(r, 0, T);
            c.rec[j] = metal_coef(r, 1, T);
            c.cxi[j] = metal_coef(r, 2, T);
            c.cxr[j] = metal_coef(r, 3, T);
        }
    }
}

// The T table: ln max(coefficient, 1e-300) at every node.
static __global__ void k_metal_ttable(const MetalDev m, double* out) {
    const long long total = (long long)m.ntr * 4 * m.tnt;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % m.tnt);
        const int c = (int)((q / m.tnt) % 4);
        const int j = (int)(q / (4LL * m.tnt));
        const double T = exp(m.tu0 + (double)i * m.tdu);
        out[q] = log(fmax(metal_coef(m.tr[j], c, T), 1.0e-300));
    }
}

// The line-cooling fit table: ln max(sum_k A_k exp(-T_k/T) / sqrt(T), 1e-300)
// of every stage at every node (cooling_mod.f90:98-122 fits).
static __global__ void k_metal_ctable(const MetalDev m, double* out) {
    const long long total = (long long)m.nst * m.tnt;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % m.tnt);
        const int s = (int)(q / m.tnt);
        const double T = exp(m.tu0 + (double)i * m.tdu);
        const MetalStage& st = m.st[s];
        double fit = 0.0;
        for (int k = 0; k < st.nterm; ++k) fit = fit + st.A[k] * exp(-st.Ti[k] / T);
        fit = fit * (1.0 / sqrt(T));
        out[q] = log(fmax(fit, 1.0e-300));
    }
}

// Ratio chain n_{i+1}/n_i of one element from the cache; returns the stage-1
// fraction 1/s and leaves the ratios in r (species_mod.f90:591-603, 794-812).
__device__ __forceinline__ double metal_chain(const MetalCache& c, int tr0, int ns, double ne, double nHI, double nHII,
                                              double* r) {
    for (int it = 1; it <= ns - 1; ++it) {
        const int j = tr0 + it - 1;
        double rion = c.gam[j] + ne * c.ci[j];
        if (c.cxi[j] > 0.0) rion = rion + nHII * c.cxi[j];
        double rrec = ne * c.rec[j];
        if (c.cxr[j] > 0.0) rrec = rrec + nHI * c.cxr[j];
        r[it - 1] = rion / fmax(rrec, kTinest);
    }
    double s = 1.0, prod = 1.0;
    for (int i = 1; i <= ns - 1; ++i) {
        prod = prod * r[i - 1];
        s = s + prod;
    }
    return 1.0 / s;
}

// species_metal_sums (species_mod.f90:566-614): metal electrons and the two
// charge-exchange rates hydrogen sees, from one walk of each chain.
static __device__ __noinline__ void metal_sums(const MetalDev& m, const MetalCache& c, double nH, double ne, double nHI,
                                        double nHII, double& nem_out, double& rin_out, double& rout_out) {
    // accumulated in registers, stored once (the outputs live in the caller's frame)
    double nem = 0.0, rin = 0.0, rout = 0.0;
    double r[kMaxSt];
    for (int ie = 0; ie < m.nel; ++ie) {
        const MetalEl e = m.el[ie];
        const int ns = e.nstage;
        double fr = metal_chain(c, e.tr0, ns, ne, nHI, nHII, r);
        const double nX = e.abund * nH;
        if (ns > 1) rin = rin + c.cxi[e.tr0] * nX * fr;
        for (int i = 2; i <= ns; ++i) {
            fr = fr * r[i - 2];
            nem = nem + e.abund * nH * fr * (double)(i - 1);
            rout = rout + c.cxr[e.tr0 + i - 2] * nX * fr;
            if (i < ns) rin = rin + c.cxi[e.tr0 + i - 1] * nX * fr;
        }
    }
    nem_out = nem;
    rin_out = rin;
    rout_out = rout;
}

// hydrogen_neutral_fraction (ion_balance_mod.f90:177-208): Illinois false
// position for x_HI on [0, 1] with the charge-exchange terms re-evaluated at
// every trial x.  Cas is the metal cascade at the cell's temperature: a
// type with sums(nH, ne, nHI, nHII, nem, rin, rout) (species_metal_sums) --
// SerialCascade below (one thread per leaf) or WarpCascade (one warp per
// leaf, cascade_warp.cuh).
template <class Cas>
static __device__ __noinline__ double hydrogen_neutral_fraction(const Cas& cas, double nH, double ne, double A,
                                                                double B, int* nsum) {
    double nem, rin, rout;
    *nsum += 2;
    double xa = 0.0;
    cas.sums(nH, ne, 0.0, nH, nem, rin, rout);
    double Ra = -(A + rin);
    double xb = 1.0;
    cas.sums(nH, ne, nH, 0.0, nem, rin, rout);
    double Rb = B + rout;
    const double scale = A + B + fabs(Ra) + fabs(Rb);
    double x = xb;
    for (int k = 1; k <= 80; ++k) {
        if (Rb == Ra) break;
        x = xb - Rb * (xb - xa) / (Rb - Ra);
        x = fmin(fmax(x, fmin(xa, xb)), fmax(xa, xb));
        cas.sums(nH, ne, nH * x, nH * (1.0 - x), nem, rin, rout);
        ++*nsum;
        const double Rx = x * (B + rin + rout) - (A + rin);
        if (fabs(Rx) <= 1.0e-15 * scale) break;
        if (fabs(xb - xa) <= 1.0e-15) break;
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

// Verdict on one substitution step x -> xn of the warm H root with residual
// R(x) and scale sc: 1 converged (|R| <= 1e-15 sc as the Illinois iteration
// stops, or the step within rounding of x), 2 not contracting (|R| did not
// fall below prev) while the step is still above 1e-12 x, 0 step on.
__device__ __forceinline__ int h_subst_verdict(double x, double xn, double Rx, double sc, double prev) {
    if (fabs(Rx) <= 1.0e-15 * sc || fabs(xn - x) <= 1.0e-15 || fabs(xn - x) <= 4.0e-16 * x) return 1;
    if (!(fabs(Rx) < prev)) return fabs(xn - x) <= 1.0e-12 * x ? 1 : 2;
    return 0;
}

// The same root from a warm start xg (the bracketed cell solve): the
// substitution x <- (A + rin(x)) / (B + rin(x) + rout(x)), whose fixed point
// is the root of R(x) = x (B + rin + rout) - (A + rin), while |R| falls,
// stopping on h_subst_verdict; Illinois on [0, 1] when the steps stop
// contracting or do not settle in 8 steps.  *nem_x: the metal electrons
// of the sums at the returned x.
template <class Cas>
static __device__ __noinline__ double hydrogen_neutral_fraction_warm(const Cas& cas, double nH, double ne, double A,
                                                                     double B, double xg, int* nsum, double* nem_x) {
    double x = fmin(fmax(xg, 0.0), 1.0);
    double prev = 1.0e300;
    for (int k = 0; k < 8; ++k) {
        double nem, rin, rout;
        cas.sums(nH, ne, nH * x, nH * (1.0 - x), nem, rin, rout);
        ++*nsum;
        const double Rx = x * (B + rin + rout) - (A + rin);
        const double scale = A + B + fabs(A + rin) + fabs(B + rout);
        const double xn = fmin(fmax((A + rin) / (B + rin + rout), 0.0), 1.0);
        const int v = h_subst_verdict(x, xn, Rx, scale, prev);
        if (v == 1) {
            *nem_x = nem;
            return x;
        }
        if (v == 2) break;   // not contracting: bracket instead
        prev = fabs(Rx);
        x = xn;
    }
    x = hydrogen_neutral_fraction(cas, nH, ne, A, B, nsum);
    double rin, rout;
    cas.sums(nH, ne, nH * x, nH * (1.0 - x), *nem_x, rin, rout);
    ++*nsum;
    return x;
}

// charge_neutrality_ne (ion_balance_mod.f90:235-253) with the cascade
// already prepared at the written temperature.
template <class Cas>
static __device__ __noinline__ double charge_neutrality_ne(const Cas& cas, double nH, double ne_HHe, double xHI,
                                                           double ne_seed) {
    const double nHI = nH * xHI, nHII = nH * (1.0 - xHI);
    double ne = fmax(ne_seed, 1.0e-12 * nH);
    for (int it = 1; it <= 200; ++it) {
        const double ne_old = ne;
        double nem, rin, rout;
        cas.sums(nH, ne_old, nHI, nHII, nem, rin, rout);
        ne = ne_HHe + nem;
        ne = fmax(0.5 * (ne + ne_old), 1.0e-12 * nH);
        if (fabs(ne - ne_old) <= 1.0e-10 * ne) break;
    }
    return ne;
}

// species_stage_cache_refresh (species_mod.f90:247-261) for one leaf, stored
// as the opacity weight n_H A_el f_it * colscale of each transition in
// threshold order (the factor species_cached_opacity applies per packet).
template <typename R>
static __device__ __noinline__ void metal_opacity_fill(const MetalDev& m, const MetalCache& c, long long il, double nH,
                                                double ne, double xHI, double colscale) {
    R* o = static_cast<R*>(m.opac) + il * m.ntrp;
    double r[kMaxSt];
    const double nHI = nH * xHI, nHII = nH * (1.0 - xHI);
    for (int ie = 0; ie < m.nel; ++ie) {
        const MetalEl e = m.el[ie];
        double fr = metal_chain(c, e.tr0, e.nstage, ne, nHI, nHII, r);
        for (int it = 1; it <= e.nstage - 1; ++it) {
            if (it > 1) fr = fr * r[it - 2];
            const MetalTr& t = m.tr[e.tr0 + it - 1];
            o[t.flat] = (R)(nH * (e.abund * fr) * colscale);
        }
    }
}

// The cascade of one leaf held by one thread: the (leaf, T) rate cache.
struct SerialCascade {
    const MetalDev* m;
    MetalCache c;
    __device__ void prepare(long long il, double T) { metal_prepare(*m, il, T, c); }
    __device__ void sums(double nH, double ne, double nHI, double nHII, double& nem, double& rin, double& rout) const {
        metal_sums(*m, c, nH, ne, nHI, nHII, nem, rin, rout);
    }
    template <typename R>
    __device__ void opacity_fill(long long il, double nH, double ne, double xHI, double colscale) const {
        metal_opacity_fill<R>(*m, c, il, nH, ne, xHI, colscale);
    }
};

// The four metal terms of net_rate (thermal_mod.f90:53-71): line cooling
// (fits with the n-level suppression), H-impact [C II] 158 um / [O I] 63 um,
// net-charge free-free and photoheating, at one (T, n_e, x_HI).
struct MetalThermalTerms {
    double cool, cool_H, freefree, heat;
};

}  // namespace mochii
