// Per-leaf ionisation balance at fixed T_e and the absorber-column refresh.
//
// k_balance restates gas_equilibrium_update (ion_balance_mod.f90:352-434):
// one thread per leaf runs solve_ion_cell (ion_balance_mod.f90:53-150, the
// damped n_e fixed point with closed-form x_HI and the He ratio chain, at
// most 200 passes), under-relaxes toward the solution, rebuilds n_e, and
// refreshes the leaf's absorber columns for the next transport pass
// (gas_opacity_fill, gas_opacity_mod.f90:299, fused here).  Convergence
// measures are reduced per block in a fixed order and summed on the host,
// so the metrics are deterministic.
#include <cuda_runtime.h>

#include "ctx.h"
#include "physics.cuh"
#include "thermal.h"
#include "transport.h"

namespace mochii {

namespace {

constexpr int kBThreads = 256;

// Temperature-dependent coefficients of the balance: recombination
// (case A or B) and collisional ionisation of H I, He I, He II.
struct Coef {
    double aH, aHe2, aHe3, cH, cHe1, cHe2;
};

struct BalArgs {
    const double* nH;
    double* xHI;
    double* xHeI;
    double* xHeII;
    double* ne;
    double* Te;
    const double* rates;   // gamma_HI, gamma_HeI, gamma_HeII, heat_* (6 x nleaf)
    void* col;
    double* partial;
    unsigned long long* counters;
    long long nleaf;
    double T, yHe, relax, colscale, vol;
    RateSel rs;
    Coef k;   // coefficients at the fixed temperature (equilibrium update)
    int caseA, nabs, fp32;
};

// Absorber columns n_i * distance2cm * 1e-18 for one leaf.
__device__ __forceinline__ void write_columns(void* col, long long il, int nabs, int fp32, double nH, double yHe,
                                              double xHI, double xHeI, double xHeII, double scale) {
    const double c0 = nH * xHI * scale;
    if (nabs == 1) {
        if (fp32) static_cast<float*>(col)[il] = (float)c0;
        else static_cast<double*>(col)[il] = c0;
        return;
    }
    const double c1 = nH * yHe * xHeI * scale, c2 = nH * yHe * xHeII * scale;
    if (fp32) {
        static_cast<float4*>(col)[il] = make_float4((float)c0, (float)c1, (float)c2, 0.0f);
    } else {
        double2* p = static_cast<double2*>(col) + 2 * il;
        p[0] = make_double2(c0, c1);
        p[1] = make_double2(c2, 0.0);
    }
}

__global__ void k_columns(const double* __restrict__ nH, const double* __restrict__ xHI,
                          const double* __restrict__ xHeI, const double* __restrict__ xHeII, void* col,
                          long long nleaf, int nabs, int fp32, double yHe, double scale) {
    for (long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x; il < nleaf;
         il += (long long)gridDim.x * blockDim.x)
        write_columns(col, il, nabs, fp32, nH[il], yHe, xHI[il], xHeI[il], xHeII[il], scale);
}

__host__ __device__ Coef coef_at(const RateSel& rs, int caseA, double T) {
    Coef k;
    k.aH = caseA ? alphaA_HII(rs, T) : alphaB_HII(rs, T);
    k.aHe2 = caseA ? alphaA_HeII(rs, T) : alphaB_HeII(rs, T);
    k.aHe3 = caseA ? alphaA_HeIII(rs, T) : alphaB_HeIII(rs, T);
    k.cH = ci_HI(rs, T);
    k.cHe1 = ci_HeI(rs, T);
    k.cHe2 = ci_HeII(rs, T);
    return k;
}

// The out-of-line copy the thermal kernel calls once per trial temperature
// (keeps the FP64 pow/exp bodies out of the solver loop's registers).
__device__ __noinline__ Coef coef_at_call(const RateSel& rs, int caseA, double T) { return coef_at(rs, caseA, T); }

// solve_ion_cell on the H/He path (ion_balance_mod.f90:53-150; no metal
// electrons, no charge exchange, so the closed-form substitution branch):
// returns the number of fixed-point passes used.
__device__ int solve_cell(const Coef& k, double yHe, double gH, double gHe1, double gHe2, double nH, double& xHI,
                          double& xHeI, double& xHeII, double& ne) {
    double xHeIII = fmax(0.0, 1.0 - xHeI - xHeII);
    ne = nH * ((1.0 - xHI) + yHe * (xHeII + 2.0 * xHeIII));
    ne = fmax(ne, 1.0e-12 * nH);
    int it = 1;
    for (; it <= 200; ++it) {
        const double ne_old = ne;
        const double denH = gH + (k.cH + k.aH) * ne + 0.0 + 0.0;
        xHI = denH > 0.0 ? (k.aH * ne + 0.0) / denH : 1.0;
        const double r1 = fmin((gHe1 + k.cHe1 * ne) / (k.aHe2 * ne), 1.0e150);
        const double r2 = fmin((gHe2 + k.cHe2 * ne) / (k.aHe3 * ne), 1.0e150);
        xHeI = 1.0 / (1.0 + r1 + r1 * r2);
        xHeII = xHeI * r1;
        xHeIII = xHeII * r2;
        ne = nH * ((1.0 - xHI) + yHe * (xHeII + 2.0 * xHeIII));
        ne = fmax(0.5 * (ne + ne_old), 1.0e-12 * nH);
        if (fabs(ne - ne_old) <= 1.0e-10 * ne) break;
    }
    return it;
}

__global__ void __launch_bounds__(kBThreads) k_balance(const BalArgs a) {
    __shared__ double sh[3][kBThreads];
    double mdx = 0.0, sdx = 0.0, sx = 0.0;
    unsigned long long solved = 0, caps = 0;
    for (long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x; il < a.nleaf;
         il += (long long)gridDim.x * blockDim.x) {
        const double nH = a.nH[il];
        const double x0 = a.xHI[il], h10 = a.xHeI[il], h20 = a.xHeII[il];
        if (nH <= 0.0) {   // ion_balance_mod.f90:383-387
            a.ne[il] = 0.0;
            write_columns(a.col, il, a.nabs, a.fp32, nH, a.yHe, x0, h10, h20, a.colscale);
            continue;
        }
        double xHI = x0, xHeI = h10, xHeII = h20, ne;
        const int it = solve_cell(a.k, a.yHe, a.rates[il], a.rates[a.nleaf + il], a.rates[2 * a.nleaf + il], nH, xHI,
                                  xHeI, xHeII, ne);
        ++solved;
        if (it > 200) ++caps;
        const double w = a.relax;
        const double xn = (1.0 - w) * x0 + w * xHI;
        const double h1n = (1.0 - w) * h10 + w * xHeI;
        const double h2n = (1.0 - w) * h20 + w * xHeII;
        const double h3n = fmax(0.0, 1.0 - h1n - h2n);
        a.xHI[il] = xn;
        a.xHeI[il] = h1n;
        a.xHeII[il] = h2n;
        a.ne[il] = nH * ((1.0 - xn) + a.yHe * (h2n + 2.0 * h3n));
        write_columns(a.col, il, a.nabs, a.fp32, nH, a.yHe, xn, h1n, h2n, a.colscale);
        const double dx = fabs(xn - x0);
        mdx = fmax(mdx, dx);
        sdx = sdx + a.vol * dx;
        sx = sx + a.vol * (1.0 - xn);
    }
    const int t = threadIdx.x;
    sh[0][t] = mdx;
    sh[1][t] = sdx;
    sh[2][t] = sx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (t < s) {
            sh[0][t] = fmax(sh[0][t], sh[0][t + s]);
            sh[1][t] = sh[1][t] + sh[1][t + s];
            sh[2][t] = sh[2][t] + sh[2][t + s];
        }
        __syncthreads();
    }
    if (t == 0) {
        a.partial[3 * blockIdx.x + 0] = sh[0][0];
        a.partial[3 * blockIdx.x + 1] = sh[1][0];
        a.partial[3 * blockIdx.x + 2] = sh[2][0];
    }
    for (int o = 16; o > 0; o >>= 1) {
        solved += __shfl_down_sync(0xffffffffu, solved, o);
        caps += __shfl_down_sync(0xffffffffu, caps, o);
    }
    if ((t & 31) == 0) {
        if (solved) atomicAdd(a.counters + 0, solved);
        if (caps) atomicAdd(a.counters + 1, caps);
    }
}

// ---- thermal balance (thermal_mod.f90) -------------------------------------
struct ThArgs {
    BalArgs b;
    ThermalDev td;
    double te_min, te_max;
};

// gbar_ff (cooling_mod.f90:223-234): linear in log10 T on the 41-node table.
__device__ double gbar_ff(const double* __restrict__ gff, double T, int Z) {
    const int iz = max(1, min(Z, kGffNZ));
    const double l1 = 2.0, l2 = 2.0 + 4.0 * 1.0 / (double)(kGffNT - 1), lN = 2.0 + 4.0;
    const double lt = fmin(fmax(log10(T), l1), lN);
    const int i = min((int)((lt - l1) / (l2 - l1)) + 1, kGffNT - 1);
    const double li = 2.0 + 4.0 * (double)(i - 1) / (double)(kGffNT - 1);
    const double li1 = 2.0 + 4.0 * (double)i / (double)(kGffNT - 1);
    const double w = (lt - li) / (li1 - li);
    return gff[(i - 1) * kGffNZ + iz - 1] * (1.0 - w) + gff[i * kGffNZ + iz - 1] * w;
}

// The n-level suppression of the H I line-cooling fit at (T, n_e):
// Lambda = lam_fit [f_cov S + 1 - f_cov], S = Lambda_SE(T, ne)/Lambda_SE(T, floor),
// f_cov = min(1, Lambda_SE(T, floor)/lam_fit); ln(Lambda) linear in 1/T
// inside a log-T cell and log-linear in log n_e (nlevel_cooling_mod.f90:163-271).
__device__ double nl_col(const ThermalDev& t, int it, int j, double w1, double wt) {
    const double Li = t.lamref[it - 1] * t.Ssup[(it - 1) * kNlNNE + (j - 1)];
    const double Lip = t.lamref[it] * t.Ssup[it * kNlNNE + (j - 1)];
    if (Li > 0.0 && Lip > 0.0) return exp(log(Li) + w1 * (log(Lip) - log(Li)));
    return Li * (1.0 - wt) + Lip * wt;
}

__device__ double nl_apply(const ThermalDev& t, double lam_fit, double T, double ne) {
    const double lt = fmin(fmax(log10(T), 2.0), 2.0 + 0.01 * (double)(kNlNT - 1));
    const int it = min((int)((lt - 2.0) / 0.01) + 1, kNlNT - 1);
    const double gi = 2.0 + 0.01 * (double)(it - 1), gi1 = 2.0 + 0.01 * (double)it;
    const double w1 = (1.0 / pow(10.0, lt) - t.tinv[it - 1]) / (t.tinv[it] - t.tinv[it - 1]);
    const double wt = fmin(fmax((lt - gi) / (gi1 - gi), 0.0), 1.0);
    const double lamref = nl_col(t, it, 1, w1, wt);
    const double lne = log10(ne);
    double lam;
    if (lne <= -6.0) {
        lam = lamref;
    } else if (lne >= -6.0 + 0.1 * (double)(kNlNNE - 1)) {
        lam = nl_col(t, it, kNlNNE, w1, wt);
    } else {
        const int je = min((int)((lne + 6.0) / 0.1) + 1, kNlNNE - 1);
        const double gj = -6.0 + 0.1 * (double)(je - 1), gj1 = -6.0 + 0.1 * (double)je;
        const double wn = (lne - gj) / (gj1 - gj);
        const double L0 = nl_col(t, it, je, w1, wt), L1 = nl_col(t, it, je + 1, w1, wt);
        lam = (L0 > 0.0 && L1 > 0.0) ? exp(log(L0) + wn * (log(L1) - log(L0))) : L0 * (1.0 - wn) + L1 * wn;
    }
    const double S = lam / fmax(lamref, kTinest);
    const double fcov = fmin(1.0, lamref / fmax(lam_fit, kTinest));
    return lam_fit * (fcov * S + (1.0 - fcov));
}

// cooling_total (cooling_mod.f90:240-276): recombination (Hui & Gnedin
// fits, He II as k T alpha), free-free with the net-charge Gaunt factor,
// collisional-ionisation energy loss, and H I collisional excitation.
__device__ __noinline__ double cooling_total(const ThermalDev& t, const RateSel& rs, int caseA, double yHe, double T, double nH,
                                double ne, double xHI, double xHeI, double xHeII) {
    const double xHeIII = fmax(0.0, 1.0 - xHeI - xHeII);
    const double nHI = nH * xHI, nHII = nH * (1.0 - xHI);
    const double nHeI = nH * yHe * xHeI, nHeII = nH * yHe * xHeII, nHeIII = nH * yHe * xHeIII;
    double cool;
    if (caseA) {
        cool = ne * (nHII * hg_fit(T, 157807.0, 1.778e-29 * T, 1.965, 0.541, 0.502, 2.697) +
                     nHeII * (kKboltz * T * alphaA_HeII(rs, T)) +
                     nHeIII * (2.0 * hg_fit(T, 631515.0, 1.778e-29 * T, 1.965, 0.541, 0.502, 2.697)));
    } else {
        cool = ne * (nHII * hg_fit(T, 157807.0, 3.435e-30 * T, 1.970, 2.250, 0.376, 3.720) +
                     nHeII * (kKboltz * T * alphaB_HeII(rs, T)) +
                     nHeIII * (2.0 * hg_fit(T, 631515.0, 3.435e-30 * T, 1.970, 2.250, 0.376, 3.720)));
    }
    cool = cool + 1.42554e-27 * sqrt(T) * ne * ((nHII + nHeII) * gbar_ff(t.gff, T, 1) + 4.0 * nHeIII * gbar_ff(t.gff, T, 2));
    cool = cool + ne * (nHI * ci_HI(rs, T) * kEthHI + nHeI * ci_HeI(rs, T) * kEthHeI + nHeII * ci_HeII(rs, T) * kEthHeII) * kEv2erg;
    double fit = 0.0;
    for (int i = 0; i < t.hi_nterm; ++i) fit = fit + t.hi_A[i] * exp(-t.hi_T[i] / T);
    fit = fit / sqrt(T);
    const double lam = t.use_hi_table ? nl_apply(t, fit, T, ne) : fit;
    return cool + ne * nHI * lam;
}

// net_rate (thermal_mod.f90:38-115), H/He path.
__device__ double net_rate(const ThArgs& a, long long il, double T, double nH, double& xHI, double& xHeI,
                           double& xHeII, double& ne, int* passes) {
    const BalArgs& b = a.b;
    const long long n = b.nleaf;
    const Coef k = coef_at_call(b.rs, b.caseA, T);
    *passes += solve_cell(k, b.yHe, b.rates[il], b.rates[n + il], b.rates[2 * n + il], nH, xHI, xHeI, xHeII, ne);
    const double heat = nH * (xHI * b.rates[3 * n + il] + b.yHe * (xHeI * b.rates[4 * n + il] + xHeII * b.rates[5 * n + il]));
    return heat - cooling_total(a.td, b.rs, b.caseA, b.yHe, T, nH, ne, xHI, xHeI, xHeII);
}

// gas_thermal_update (thermal_mod.f90:124-249): bisection on log T in
// [te_min, te_max] (at most 60 halvings, stop at thi/tlo - 1 < 1e-5), the
// ionisation re-solved at every trial temperature.
__global__ void __launch_bounds__(kBThreads) k_thermal(const ThArgs a) {
    __shared__ double sh[6][kBThreads];
    const BalArgs& b = a.b;
    double mdx = 0.0, mdt = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
    unsigned long long solved = 0, caps = 0;
    for (long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x; il < b.nleaf;
         il += (long long)gridDim.x * blockDim.x) {
        const double nH = b.nH[il];
        const double x0 = b.xHI[il], h10 = b.xHeI[il], h20 = b.xHeII[il], T0 = b.Te[il];
        if (nH <= 0.0) {
            b.ne[il] = 0.0;
            write_columns(b.col, il, b.nabs, b.fp32, nH, b.yHe, x0, h10, h20, b.colscale);
            continue;
        }
        double xHI = x0, xHeI = h10, xHeII = h20, ne = 0.0;
        int passes = 0;
        double tlo = a.te_min, thi = a.te_max, te;
        const double net_lo = net_rate(a, il, tlo, nH, xHI, xHeI, xHeII, ne, &passes);
        const double net_hi = net_rate(a, il, thi, nH, xHI, xHeI, xHeII, ne, &passes);
        if (net_lo <= 0.0) {
            te = tlo;
        } else if (net_hi >= 0.0) {
            te = thi;
        } else {
            for (int it = 1; it <= 60; ++it) {
                const double tmid = sqrt(tlo * thi);
                const double nm = net_rate(a, il, tmid, nH, xHI, xHeI, xHeII, ne, &passes);
                if (nm > 0.0) tlo = tmid; else thi = tmid;
                if (thi / tlo - 1.0 < 1.0e-5) break;
            }
            te = sqrt(tlo * thi);
        }
        int last = 0;
        net_rate(a, il, te, nH, xHI, xHeI, xHeII, ne, &last);
        ++solved;
        if (last > 200) ++caps;
        const double w = b.relax;
        const double xn = (1.0 - w) * x0 + w * xHI;
        const double h1n = (1.0 - w) * h10 + w * xHeI;
        const double h2n = (1.0 - w) * h20 + w * xHeII;
        const double h3n = fmax(0.0, 1.0 - h1n - h2n);
        const double nen = nH * ((1.0 - xn) + b.yHe * (h2n + 2.0 * h3n));
        b.xHI[il] = xn;
        b.xHeI[il] = h1n;
        b.xHeII[il] = h2n;
        b.ne[il] = nen;
        b.Te[il] = te;
        write_columns(b.col, il, b.nabs, b.fp32, nH, b.yHe, xn, h1n, h2n, b.colscale);
        const double dx = fabs(xn - x0);
        mdx = fmax(mdx, dx);
        mdt = fmax(mdt, fabs(te - T0) / T0);
        s1 = s1 + b.vol * dx;
        s2 = s2 + b.vol * (1.0 - xn);
        s3 = s3 + b.vol * nen * fabs(te - T0);
        s4 = s4 + b.vol * nen * te;
    }
    const int t = threadIdx.x;
    sh[0][t] = mdx; sh[1][t] = mdt; sh[2][t] = s1; sh[3][t] = s2; sh[4][t] = s3; sh[5][t] = s4;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (t < s) {
            sh[0][t] = fmax(sh[0][t], sh[0][t + s]);
            sh[1][t] = fmax(sh[1][t], sh[1][t + s]);
            for (int k = 2; k < 6; ++k) sh[k][t] = sh[k][t] + sh[k][t + s];
        }
        __syncthreads();
    }
    if (t == 0)
        for (int k = 0; k < 6; ++k) b.partial[6 * blockIdx.x + k] = sh[k][0];
    for (int o = 16; o > 0; o >>= 1) {
        solved += __shfl_down_sync(0xffffffffu, solved, o);
        caps += __shfl_down_sync(0xffffffffu, caps, o);
    }
    if ((t & 31) == 0) {
        if (solved) atomicAdd(b.counters + 0, solved);
        if (caps) atomicAdd(b.counters + 1, caps);
    }
}

int nblocks(long long work, int threads, int cap) {
    long long b = (work + threads - 1) / threads;
    return (int)(b < 1 ? 1 : b > cap ? cap : b);
}

}  // namespace

int balance_blocks(const mochii_ctx* c) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    return nblocks(c->grid.nleaf, kBThreads, sms * 8);
}

cudaError_t launch_columns(mochii_ctx* c) {
    k_columns<<<nblocks(c->grid.nleaf, 256, 148 * 16), 256, 0, c->stream>>>(
        c->nH, c->xHI, c->xHeI, c->xHeII, c->col, c->grid.nleaf, c->nabs, c->fp32 ? 1 : 0, c->par.He_abund,
        c->par.distance2cm * 1.0e-18);
    return cudaGetLastError();
}

static BalArgs bal_args(mochii_ctx* c) {
    BalArgs a;
    a.nH = c->nH;
    a.xHI = c->xHI;
    a.xHeI = c->xHeI;
    a.xHeII = c->xHeII;
    a.ne = c->ne;
    a.Te = c->Te;
    a.rates = c->rates;
    a.col = c->col;
    a.partial = c->bw.partial;
    a.counters = c->bw.counters;
    a.nleaf = c->grid.nleaf;
    a.T = c->par.te_fixed;
    a.yHe = c->par.He_abund;
    a.relax = c->par.ion_relax;
    a.colscale = c->par.distance2cm * 1.0e-18;
    const double w = c->grid.dcell;   // (2*leaf_half)^3 on the uniform grid
    a.vol = w * w * w;
    a.rs.hui_gnedin = c->par.recomb_hui_gnedin;
    a.rs.dere_hybrid = c->par.ci_dere_hybrid;
    a.caseA = c->par.caseA;
    a.nabs = c->nabs;
    a.fp32 = c->fp32 ? 1 : 0;
    a.k = coef_at(a.rs, a.caseA, a.T);   // fixed T: evaluated once on the host
    return a;
}

cudaError_t launch_balance(mochii_ctx* c) {
    const BalArgs a = bal_args(c);
    k_balance<<<c->bw.blocks, kBThreads, 0, c->stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_thermal(mochii_ctx* c) {
    ThArgs a;
    a.b = bal_args(c);
    a.td = c->th;
    a.te_min = c->par.te_min;
    a.te_max = c->par.te_max;
    k_thermal<<<c->bw.blocks, kBThreads, 0, c->stream>>>(a);
    return cudaGetLastError();
}

}  // namespace mochii
