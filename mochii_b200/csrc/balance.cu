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
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>

#include "ctx.h"
#include "metals.cuh"
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
    const double4* lg;                // octree leaf geometry (per-leaf volume), null on the Cartesian grid
    const double* rhokap;             // grey dust opacity per leaf, null without grains
    RateSel rs;
    Coef k;   // coefficients at the fixed temperature (equilibrium update)
    int caseA, nabs, fp32;
    MetalDev m;                       // trace metals; m.ntr == 0 without
    int metal_ne, two_way, metal_heat, metal_ff;
    int fast;                         // bracketed Illinois solves (solver_bracketed)
    double nemax;                     // largest n_e per n_H: 1 + 2 y_He + metal electrons
};

// Volume weight of a leaf in the convergence sums: (2 leaf_half)^3.
__device__ __forceinline__ double leaf_vol(const BalArgs& a, long long il) {
    if (!a.lg) return a.vol;
    const double w = 2.0 * a.lg[il].w;
    return w * w * w;
}

// Absorber columns n_i * distance2cm * 1e-18 for one leaf; the fourth
// slot of the 4-wide layout holds the grey dust opacity per code length
// rhokap (0 without grains).
__device__ __forceinline__ void write_columns(void* col, long long il, int nabs, int fp32, double nH, double yHe,
                                              double xHI, double xHeI, double xHeII, double scale, double rk) {
    const double c0 = nH * xHI * scale;
    if (nabs == 1) {
        if (fp32) static_cast<float*>(col)[il] = (float)c0;
        else static_cast<double*>(col)[il] = c0;
        return;
    }
    const double c1 = nH * yHe * xHeI * scale, c2 = nH * yHe * xHeII * scale;
    if (fp32) {
        static_cast<float4*>(col)[il] = make_float4((float)c0, (float)c1, (float)c2, (float)rk);
    } else {
        double2* p = static_cast<double2*>(col) + 2 * il;
        p[0] = make_double2(c0, c1);
        p[1] = make_double2(c2, rk);
    }
}

// The metal opacity weights of one leaf at its written state (T_e, n_e, x_HI).
__device__ __noinline__ void metal_fill_at(const MetalDev& m, MetalCache& mc, long long il, double T, double nH,
                                           double ne, double xHI, double scale, int fp32) {
    metal_prepare(m, il, T, mc);
    if (fp32) metal_opacity_fill<float>(m, mc, il, nH, ne, xHI, scale);
    else metal_opacity_fill<double>(m, mc, il, nH, ne, xHI, scale);
}

// gas_opacity_fill (gas_opacity_mod.f90:299-306): absorber columns and, with
// metals, the stage-fraction opacity weights (species_stage_cache_refresh).
__global__ void k_columns(const double* __restrict__ nH, const double* __restrict__ xHI,
                          const double* __restrict__ xHeI, const double* __restrict__ xHeII,
                          const double* __restrict__ ne, const double* __restrict__ Te, void* col,
                          long long nleaf, int nabs, int fp32, double yHe, double scale, const MetalDev m,
                          const double* __restrict__ rhokap) {
    for (long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x; il < nleaf;
         il += (long long)gridDim.x * blockDim.x) {
        write_columns(col, il, nabs, fp32, nH[il], yHe, xHI[il], xHeI[il], xHeII[il], scale,
                      rhokap ? rhokap[il] : 0.0);
        if (m.ntr > 0) {
            MetalCache mc;
            metal_fill_at(m, mc, il, Te[il], nH[il], ne[il], xHI[il], scale, fp32);
        }
    }
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

// solve_ion_cell with the metal cascade (ion_balance_mod.f90:53-150): metal
// electrons join the n_e closure (metal_ne), and with the two-way charge
// exchange x_HI is the root of hydrogen's balance at each n_e
// (hydrogen_neutral_fraction); the cache mc is prepared at T.
template <class Cas>
__device__ __noinline__ int solve_cell_metal(const Coef& k, double yHe, double gH, double gHe1, double gHe2, double nH,
                                             double& xHI, double& xHeI, double& xHeII, double& ne, const Cas& mc,
                                             int with_ne, int with_cx, int* nsum) {
    double xHeIII = fmax(0.0, 1.0 - xHeI - xHeII);
    ne = nH * ((1.0 - xHI) + yHe * (xHeII + 2.0 * xHeIII));
    ne = fmax(ne, 1.0e-12 * nH);
    double nem = 0.0, rin = 0.0, rout = 0.0;
    int it = 1;
    for (; it <= 200; ++it) {
        const double ne_old = ne;
        if (with_ne || with_cx) {
            mc.sums(nH, ne_old, nH * xHI, nH * (1.0 - xHI), nem, rin, rout);
            ++*nsum;
            if (!with_cx) {
                rin = 0.0;
                rout = 0.0;
            }
        }
        if (with_cx) {
            xHI = hydrogen_neutral_fraction(mc, nH, ne, k.aH * ne, gH + (k.cH + k.aH) * ne, nsum);
        } else {
            const double denH = gH + (k.cH + k.aH) * ne + rin + rout;
            xHI = denH > 0.0 ? (k.aH * ne + rin) / denH : 1.0;
        }
        const double r1 = fmin((gHe1 + k.cHe1 * ne) / (k.aHe2 * ne), 1.0e150);
        const double r2 = fmin((gHe2 + k.cHe2 * ne) / (k.aHe3 * ne), 1.0e150);
        xHeI = 1.0 / (1.0 + r1 + r1 * r2);
        xHeII = xHeI * r1;
        xHeIII = xHeII * r2;
        ne = nH * ((1.0 - xHI) + yHe * (xHeII + 2.0 * xHeIII));
        if (with_ne) ne = ne + nem;
        ne = fmax(0.5 * (ne + ne_old), 1.0e-12 * nH);
        if (fabs(ne - ne_old) <= 1.0e-10 * ne) break;
    }
    return it;
}

// ---- bracketed solves (solver_bracketed) -----------------------------------
// The reference's damped iteration converges to the n_e at which the
// electrons the cell releases equal n_e, F(n_e) = n_e, with x_HI the root of
// hydrogen's balance at that n_e and the metal cascade evaluated there.  The
// bracketed solve finds the same root of h(n_e) = F(n_e) - n_e directly:
// geometric bracketing from the cell's current n_e, then safeguarded false
// position in ln n_e, to |h| <= 2e-10 n_e (the reference stops its damped
// steps h/2 at 1e-10 n_e).
struct CellState {
    double x, h1, h2;
};

//
// xg: a guess of x_HI (the previous evaluation's), from which the H root
// with charge exchange is found (hydrogen_neutral_fraction_warm).
template <class Cas>
__device__ __noinline__ double cell_electrons(const Coef& k, double yHe, double gH, double gHe1, double gHe2, double nH,
                                              double ne, bool metals, const Cas& mc, int with_ne, int with_cx,
                                              int* nsum, CellState& o, double xg) {
    double nem_x = 0.0;
    bool have_nem = false;
    if (metals && with_cx) {
        o.x = hydrogen_neutral_fraction_warm(mc, nH, ne, k.aH * ne, gH + (k.cH + k.aH) * ne, xg, nsum, &nem_x);
        have_nem = true;
    } else {
        const double denH = gH + (k.cH + k.aH) * ne;
        o.x = denH > 0.0 ? (k.aH * ne) / denH : 1.0;
    }
    const double r1 = fmin((gHe1 + k.cHe1 * ne) / (k.aHe2 * ne), 1.0e150);
    const double r2 = fmin((gHe2 + k.cHe2 * ne) / (k.aHe3 * ne), 1.0e150);
    o.h1 = 1.0 / (1.0 + r1 + r1 * r2);
    o.h2 = o.h1 * r1;
    const double h3 = o.h2 * r2;
    double nen = nH * ((1.0 - o.x) + yHe * (o.h2 + 2.0 * h3));
    if (metals && with_ne) {
        if (!have_nem) {
            double rin, rout;
            mc.sums(nH, ne, nH * o.x, nH * (1.0 - o.x), nem_x, rin, rout);
            ++*nsum;
        }
        nen = nen + nem_x;
    }
    return nen;
}

// Returns the number of F evaluations.
template <class Cas>
__device__ __noinline__ int solve_cell_fast(const Coef& k, double yHe, double gH, double gHe1, double gHe2, double nH,
                                            double& xHI, double& xHeI, double& xHeII, double& ne, bool metals,
                                            const Cas& mc, int with_ne, int with_cx, int* nsum, double nemax) {
    const double floor = 1.0e-12 * nH, top = nemax * nH;
    const double xHeIII = fmax(0.0, 1.0 - xHeI - xHeII);
    double a = ne > floor ? ne : fmax(nH * ((1.0 - xHI) + yHe * (xHeII + 2.0 * xHeIII)), floor);
    a = fmin(a, top);
    int nev = 0;
    CellState ea, eb, ec;
    double fa = cell_electrons(k, yHe, gH, gHe1, gHe2, nH, a, metals, mc, with_ne, with_cx, nsum, ea, xHI) - a;
    ++nev;
    double b = a, fb = fa;
    eb = ea;
    ec = ea;   // ec.x: the guess of the next evaluation's H root
    bool done = fabs(fa) <= 2.0e-10 * a;
    auto F = [&](double c, CellState& st) {
        ++nev;
        return cell_electrons(k, yHe, gH, gHe1, gHe2, nH, c, metals, mc, with_ne, with_cx, nsum, st, ec.x) - c;
    };
    // search from the warm start: the undamped fixed-point step n_e <- F(n_e),
    // then secant steps in ln n_e while |h| falls and the root stays ahead,
    // else geometric steps (x4, then squared) toward the root, until h
    // changes sign; on a clamp with h still of the same sign the damped
    // iteration would sit there
    if (!done) {
        double c = fa > 0.0 ? fmin(a + fa, top) : fmax(a + fa, floor);
        if (!(c > 0.0)) c = floor;
        double fac = 4.0;
        while (nev < 60) {
            const double fc = F(c, ec);
            b = c; fb = fc; eb = ec;
            if (fabs(fc) <= 2.0e-10 * c || fc == 0.0) {
                done = true;
                break;
            }
            if ((fc > 0.0) != (fa > 0.0)) break;            // bracketed by [a, c]
            if (c >= top || c <= floor) {
                done = true;
                break;
            }
            const double la = log(a), lc = log(c);
            double ld = lc - fc * (lc - la) / (fc - fa);     // secant in ln n_e
            const bool ahead = fc > 0.0 ? ld > lc : ld < lc;
            const double lim = log(fac);
            if (!(fabs(fc) < fabs(fa)) || !ahead || !(fabs(ld - lc) <= lim)) ld = fc > 0.0 ? lc + lim : lc - lim;
            a = c; fa = fc; ea = ec;
            c = fc > 0.0 ? fmin(exp(ld), top) : fmax(exp(ld), floor);
            fac = fac * fac;
        }
    }
    // Anderson-Bjorck false position in ln n_e on the bracket [a, b]
    if (!done) {
        double la = log(a), lb = log(b);
        int side = 0;
        for (int it = 0; it < 100 && nev < 160; ++it) {
            const double width = fabs(lb - la);
            if (width <= 1.0e-13) break;
            double lc = (la * fb - lb * fa) / (fb - fa);
            if (!(fabs(lc - la) > 1.0e-3 * width && fabs(lc - lb) > 1.0e-3 * width)) lc = 0.5 * (la + lb);
            const double c = exp(lc);
            const double fc = F(c, ec);
            b = c;          // the returned point is the last one evaluated
            eb = ec;
            if (fabs(fc) <= 2.0e-10 * c || fc == 0.0) break;
            if ((fc > 0.0) == (fb > 0.0)) {   // c replaces the b end
                if (side == -1) {
                    const double m = 1.0 - fc / fb;
                    fa = fa * (m > 0.0 ? m : 0.5);
                }
                lb = lc; fb = fc; side = -1;
            } else {                          // c replaces the a end
                if (side == +1) {
                    const double m = 1.0 - fc / fa;
                    fb = fb * (m > 0.0 ? m : 0.5);
                }
                la = lc; fa = fc; side = +1;
            }
        }
    }
    ne = b;
    xHI = eb.x;
    xHeI = eb.h1;
    xHeII = eb.h2;
    return nev;
}

__global__ void __launch_bounds__(kBThreads) k_balance(const BalArgs a) {
    __shared__ double sh[3][kBThreads];
    double mdx = 0.0, sdx = 0.0, sx = 0.0;
    unsigned long long solved = 0, caps = 0, passes = 0, sums = 0;
    for (long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x; il < a.nleaf;
         il += (long long)gridDim.x * blockDim.x) {
        const double nH = a.nH[il];
        const double x0 = a.xHI[il], h10 = a.xHeI[il], h20 = a.xHeII[il];
        if (nH <= 0.0) {   // ion_balance_mod.f90:383-387
            a.ne[il] = 0.0;
            write_columns(a.col, il, a.nabs, a.fp32, nH, a.yHe, x0, h10, h20, a.colscale, a.rhokap ? a.rhokap[il] : 0.0);
            continue;
        }
        double xHI = x0, xHeI = h10, xHeII = h20, ne;
        SerialCascade mc;
        mc.m = &a.m;
        int it, nsum = 0;
        if (a.fast) {
            if (a.m.ntr > 0) mc.prepare(il, a.T);
            ne = a.ne[il];
            it = solve_cell_fast(a.k, a.yHe, a.rates[il], a.rates[a.nleaf + il], a.rates[2 * a.nleaf + il], nH, xHI,
                                 xHeI, xHeII, ne, a.m.ntr > 0, mc, a.metal_ne, a.two_way, &nsum, a.nemax);
        } else if (a.m.ntr > 0) {
            mc.prepare(il, a.T);
            it = solve_cell_metal(a.k, a.yHe, a.rates[il], a.rates[a.nleaf + il], a.rates[2 * a.nleaf + il], nH, xHI,
                                  xHeI, xHeII, ne, mc, a.metal_ne, a.two_way, &nsum);
        } else {
            it = solve_cell(a.k, a.yHe, a.rates[il], a.rates[a.nleaf + il], a.rates[2 * a.nleaf + il], nH, xHI, xHeI,
                            xHeII, ne);
        }
        ++solved;
        if (it > 200) ++caps;
        passes += (unsigned long long)min(it, 200);
        sums += (unsigned long long)nsum;
        const double w = a.relax;
        const double xn = (1.0 - w) * x0 + w * xHI;
        const double h1n = (1.0 - w) * h10 + w * xHeI;
        const double h2n = (1.0 - w) * h20 + w * xHeII;
        const double h3n = fmax(0.0, 1.0 - h1n - h2n);
        a.xHI[il] = xn;
        a.xHeI[il] = h1n;
        a.xHeII[il] = h2n;
        double nen = nH * ((1.0 - xn) + a.yHe * (h2n + 2.0 * h3n));
        if (a.m.ntr > 0) {
            // metal electrons of the written state (ion_balance_mod.f90:401-410),
            // then the stage cache at the written T_e (gas_opacity_fill)
            if (a.metal_ne) nen = charge_neutrality_ne(mc, nH, nen, xn, ne);
            const double Tw = a.Te[il];
            if (Tw != a.T) mc.prepare(il, Tw);
            if (a.fp32) mc.opacity_fill<float>(il, nH, nen, xn, a.colscale);
            else mc.opacity_fill<double>(il, nH, nen, xn, a.colscale);
        }
        a.ne[il] = nen;
        write_columns(a.col, il, a.nabs, a.fp32, nH, a.yHe, xn, h1n, h2n, a.colscale, a.rhokap ? a.rhokap[il] : 0.0);
        const double dx = fabs(xn - x0);
        const double vol = leaf_vol(a, il);
        mdx = fmax(mdx, dx);
        sdx = sdx + vol * dx;
        sx = sx + vol * (1.0 - xn);
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
        passes += __shfl_down_sync(0xffffffffu, passes, o);
        sums += __shfl_down_sync(0xffffffffu, sums, o);
    }
    if ((t & 31) == 0) {
        if (solved) atomicAdd(a.counters + 0, solved);
        if (caps) atomicAdd(a.counters + 1, caps);
        if (passes) atomicAdd(a.counters + 2, passes);
        if (sums) atomicAdd(a.counters + 3, sums);
        if (solved) atomicAdd(a.counters + 4, solved);
    }
}

// ---- thermal balance (thermal_mod.f90) -------------------------------------
struct ThArgs {
    BalArgs b;
    ThermalDev td;
    double te_min, te_max;
    const double* Twarm;   // bracketed solve: warm-start T_e per leaf (nullptr: the current T_e)
    double tfac0;          // bracketed solve: the first bracketing step in T (1.05; smaller after a learned warm start)
    double gate;           // bracketed solve: residual gate of a learned warm start (0: none), lane layout
    const int* order;      // lockstep solve: the order to visit leaves in (nullptr: leaf order)
    unsigned* work;        // lockstep solve: cascade sums per leaf, written for the next update's order
    unsigned long long* next;   // lockstep solve: the chunk counter (warps claim 32 leaves at a time)
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
__device__ double nl_col(const double* lamref, const double* Ssup, int it, int j, double w1, double wt) {
    const double Li = lamref[it - 1] * Ssup[(it - 1) * kNlNNE + (j - 1)];
    const double Lip = lamref[it] * Ssup[it * kNlNNE + (j - 1)];
    if (Li > 0.0 && Lip > 0.0) return exp(log(Li) + w1 * (log(Lip) - log(Li)));
    return Li * (1.0 - wt) + Lip * wt;
}

// The (T, n_e) cell of the suppression tables, shared by every table at
// one (T, n_e): the log-T row it and its weights, the log-n_e column.
struct NlAt {
    int it, je, band;   // band: 0 n_e at or below the grid, 1 above it, 2 inside
    double w1, wt, wn;
};

__device__ __forceinline__ NlAt nl_at(const double* tinv, double T, double ne) {
    NlAt a;
    const double lt = fmin(fmax(log10(T), 2.0), 2.0 + 0.01 * (double)(kNlNT - 1));
    a.it = min((int)((lt - 2.0) / 0.01) + 1, kNlNT - 1);
    const double gi = 2.0 + 0.01 * (double)(a.it - 1), gi1 = 2.0 + 0.01 * (double)a.it;
    a.w1 = (1.0 / pow(10.0, lt) - tinv[a.it - 1]) / (tinv[a.it] - tinv[a.it - 1]);
    a.wt = fmin(fmax((lt - gi) / (gi1 - gi), 0.0), 1.0);
    const double lne = log10(ne);
    a.je = 1;
    a.wn = 0.0;
    if (lne <= -6.0) {
        a.band = 0;
    } else if (lne >= -6.0 + 0.1 * (double)(kNlNNE - 1)) {
        a.band = 1;
    } else {
        a.band = 2;
        a.je = min((int)((lne + 6.0) / 0.1) + 1, kNlNNE - 1);
        const double gj = -6.0 + 0.1 * (double)(a.je - 1), gj1 = -6.0 + 0.1 * (double)a.je;
        a.wn = (lne - gj) / (gj1 - gj);
    }
    return a;
}

// One column of one table at the row pair of a: ln(Lambda) linear in 1/T
// (lnL holds log(lamref * Ssup), computed once at set-up), else linear in T.
__device__ __forceinline__ double nl_col(const double* lamref, const double* Ssup, const double* lnL, const NlAt& a,
                                         int j) {
    const int it = a.it;
    const double Li = lamref[it - 1] * Ssup[(it - 1) * kNlNNE + (j - 1)];
    const double Lip = lamref[it] * Ssup[it * kNlNNE + (j - 1)];
    if (Li > 0.0 && Lip > 0.0) {
        const double li = lnL[(it - 1) * kNlNNE + (j - 1)], lip = lnL[it * kNlNNE + (j - 1)];
        return exp(li + a.w1 * (lip - li));
    }
    return Li * (1.0 - a.wt) + Lip * a.wt;
}

// The n-level suppression of a line-cooling fit at (T, n_e):
// Lambda = lam_fit [f_cov S + 1 - f_cov], S = Lambda_SE(T, ne)/Lambda_SE(T, floor),
// f_cov = min(1, Lambda_SE(T, floor)/lam_fit); ln(Lambda) linear in 1/T
// inside a log-T cell and log-linear in log n_e (nlevel_cooling_mod.f90:163-271).
__device__ __noinline__ double nl_apply(const double* lamref, const double* Ssup, const double* lnL, const NlAt& a,
                                        double lam_fit) {
    const double lref = nl_col(lamref, Ssup, lnL, a, 1);
    double lam;
    if (a.band == 0) {
        lam = lref;
    } else if (a.band == 1) {
        lam = nl_col(lamref, Ssup, lnL, a, kNlNNE);
    } else {
        const double L0 = nl_col(lamref, Ssup, lnL, a, a.je), L1 = nl_col(lamref, Ssup, lnL, a, a.je + 1);
        lam = (L0 > 0.0 && L1 > 0.0) ? exp(log(L0) + a.wn * (log(L1) - log(L0))) : L0 * (1.0 - a.wn) + L1 * a.wn;
    }
    const double S = lam / fmax(lref, kTinest);
    const double fcov = fmin(1.0, lref / fmax(lam_fit, kTinest));
    return lam_fit * (fcov * S + (1.0 - fcov));
}

// log(lamref * Ssup) of ntab tables (0 where the product is not positive).
__global__ void k_nl_log(const double* __restrict__ lamref, const double* __restrict__ Ssup, int ntab,
                         double* __restrict__ out) {
    const long long total = (long long)ntab * kNlNT * kNlNNE;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
        const long long row = q / kNlNNE;   // table * kNlNT + it
        const double L = lamref[row] * Ssup[q];
        out[q] = L > 0.0 ? log(L) : 0.0;
    }
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
    double lam = fit;
    if (t.use_hi_table) {
        const NlAt at = nl_at(t.tinv, T, ne);
        lam = nl_apply(t.lamref, t.Ssup, t.lnL, at, fit);
    }
    return cool + ne * nHI * lam;
}

// The metal terms of net_rate (thermal_mod.f90:53-71): metal_cooling
// (species_mod.f90:825-846), metal_cooling_H (:704-731), metal_freefree
// (:852-871) and metal_heating (:739-752).  One evaluation of each element's
// stage chain (from the cache at T) serves all four sums.
__device__ __noinline__ MetalThermalTerms metal_thermal(const ThermalDev& td, const MetalDev& m, const MetalCache& c,
                                                        long long il, double T, double nH, double ne, double nHI,
                                                        double nHII) {
    const double A_CII = 2.321e-6, A_OI = 8.865e-5;
    MetalThermalTerms o = {0.0, 0.0, 0.0, 0.0};
    double g[4];
    for (int z = 1; z <= 4; ++z) g[z - 1] = gbar_ff(td.gff, T, z);
    const double rsT = 1.0 / sqrt(T);
    double ff = 0.0;
    double r[kMaxSt], frac[kMaxSt];
    const NlAt at = nl_at(td.tinv, T, ne);
    for (int ie = 0; ie < m.nel; ++ie) {
        const MetalEl e = m.el[ie];
        frac[0] = metal_chain(c, e.tr0, e.nstage, ne, nHI, nHII, r);
        for (int i = 2; i <= e.nstage; ++i) frac[i - 1] = frac[i - 2] * r[i - 2];
        const double nel = e.abund * nH;
        for (int i = 1; i <= e.nstage; ++i) {
            const MetalStage& st = m.st[e.st0 + i - 1];
            if (!st.has_cool) continue;
            double fit = 0.0;
            for (int q = 0; q < st.nterm; ++q) fit = fit + st.A[q] * exp(-st.Ti[q] / T);
            fit = fit * rsT;
            const double lam = st.table >= 0 ? nl_apply(m.lamref + (size_t)st.table * kNlNT,
                                                        m.Ssup + (size_t)st.table * kNlNT * kNlNNE,
                                                        m.lnL + (size_t)st.table * kNlNT * kNlNNE, at, fit)
                                             : fit;
            o.cool = o.cool + ne * nel * frac[i - 1] * lam;
        }
        if (e.kind == 1 && e.nstage >= 2) {   // [C II] 158 um, H impact
            const double nion = e.abund * nH * frac[1];
            const double qul = 7.6e-10 * pow(T / 100.0, 0.14);
            const double qlu = 2.0 * qul * exp(-91.25 / T);
            o.cool_H = o.cool_H + nion * nHI * qlu * (91.25 * kKboltz) / (1.0 + nHI * (qul + qlu) / A_CII);
        } else if (e.kind == 2) {             // [O I] 63 um
            const double nion = e.abund * nH * frac[0];
            const double qul = 9.2e-11 * pow(T / 100.0, 0.67);
            const double qlu = 0.6 * qul * exp(-227.7 / T);
            o.cool_H = o.cool_H + nion * nHI * qlu * (227.7 * kKboltz) / (1.0 + nHI * (qul + qlu) / A_OI);
        }
        for (int j = 2; j <= e.nstage; ++j) {
            const int zion = j - 1;
            ff = ff + e.abund * frac[j - 1] * (double)(zion * zion) * g[min(zion, 4) - 1];
        }
        for (int i = 1; i <= e.nstage - 1; ++i)
            o.heat = o.heat + e.abund * nH * frac[i - 1] * m.eheat[il * m.ntr + e.tr0 + i - 1];
    }
    o.freefree = 1.42554e-27 * sqrt(T) * ne * nH * ff;
    return o;
}

__device__ __forceinline__ MetalThermalTerms thermal_terms(const ThermalDev& td, const SerialCascade& cas, long long il,
                                                         double T, double nH, double ne, double nHI, double nHII) {
    return metal_thermal(td, *cas.m, cas.c, il, T, nH, ne, nHI, nHII);
}

// ---- the metal cascade of one leaf spread over one warp ---------------------
// The thermal solve of a leaf with metals evaluates, per trial temperature,
// every transition's collisional-ionisation, recombination and charge-
// exchange coefficients and every stage's line cooling, then walks each
// element's stage chain many times (the n_e closure and the H root).  One
// thread per leaf keeps that cache in local memory and runs the leaves of a
// warp through different trial sequences.  Here one warp owns one leaf:
// lane j % 32 evaluates the coefficients of transition j and the line
// cooling of stage s (lane s % 32), element e's chain is walked by lane e
// from its own registers (its <= 5 transitions, fetched once per trial
// temperature), and the per-element sums are added in element order with
// the result in every lane.  Every lane runs the same solver control flow
// on the same values; the leaf's H/He arithmetic is repeated in all lanes.
constexpr unsigned kFull = 0xffffffffu;
constexpr int kTrSlots = (kMaxTr + 31) / 32;
constexpr int kStSlots = (kMaxEl * kMaxSt + 31) / 32;
constexpr int kEt = kMaxSt - 1;   // transitions per element

template <int S>
__device__ __forceinline__ double lane_fetch(const double (&v)[S], int j) {
    double out = 0.0;
#pragma unroll
    for (int q = 0; q < S; ++q) {
        const double x = __shfl_sync(kFull, v[q], j & 31);
        if ((j >> 5) == q) out = x;
    }
    return out;
}

struct WarpCascade {
    const MetalDev* m;
    int lane, ns, tr0, st0, kind, coolmask;
    long long il = -1;
    double abund;
    double gam[kEt], eheat[kEt], ci[kEt], rec[kEt], cxi[kEt], cxr[kEt];

    __device__ void init(const MetalDev& md) {
        m = &md;
        lane = threadIdx.x & 31;
        ns = 1; tr0 = 0; st0 = 0; kind = 0; coolmask = 0; abund = 0.0;
        if (lane < md.nel) {
            const MetalEl e = md.el[lane];
            ns = e.nstage; tr0 = e.tr0; st0 = e.st0; kind = e.kind; abund = e.abund;
            for (int i = 0; i < ns; ++i)
                if (md.st[st0 + i].has_cool) coolmask |= 1 << i;
        }
    }
    // the element's photoionisation and photoheating rates in leaf l
    __device__ void leaf(long long l) {
        il = l;
#pragma unroll
        for (int i = 0; i < kEt; ++i) {
            gam[i] = 0.0;
            eheat[i] = 0.0;
            if (i < ns - 1) {
                gam[i] = m->egam[l * m->ntr + tr0 + i];
                eheat[i] = m->eheat[l * m->ntr + tr0 + i];
            }
        }
    }
    // species_ne_prepare (species_mod.f90:517-536) at T
    __device__ void prepare(long long l, double T) {
        if (l != il) leaf(l);
        double tci[kTrSlots], trec[kTrSlots], tcxi[kTrSlots], tcxr[kTrSlots];
#pragma unroll
        for (int q = 0; q < kTrSlots; ++q) {
            const int j = lane + 32 * q;
            tci[q] = trec[q] = tcxi[q] = tcxr[q] = 0.0;
            if (j < m->ntr) {
                const MetalTr& r = m->tr[j];
                tci[q] = voronov(T, r.ci[0], r.ci[1], r.ci[2], r.ci[3], r.ci[4]) * r.cidr;
                trec[q] = metal_alpha_rec(r, T);
                tcxi[q] = r.cxi_form > 0 ? metal_cx_rate(r.cxi_form, r.cxi, T) : 0.0;
                tcxr[q] = r.cxr_form > 0 ? metal_cx_rate(r.cxr_form, r.cxr, T) : 0.0;
            }
        }
#pragma unroll
        for (int i = 0; i < kEt; ++i) {
            const int j = i < ns - 1 ? tr0 + i : 0;
            ci[i] = lane_fetch(tci, j);
            rec[i] = lane_fetch(trec, j);
            cxi[i] = lane_fetch(tcxi, j);
            cxr[i] = lane_fetch(tcxr, j);
        }
    }
    // metal_chain: ratios n_{i+1}/n_i and the stage-1 fraction
    __device__ __forceinline__ double chain(double ne, double nHI, double nHII, double (&r)[kEt]) const {
#pragma unroll
        for (int i = 0; i < kEt; ++i) {
            double rion = gam[i] + ne * ci[i];
            if (cxi[i] > 0.0) rion = rion + nHII * cxi[i];
            double rrec = ne * rec[i];
            if (cxr[i] > 0.0) rrec = rrec + nHI * cxr[i];
            r[i] = rion / fmax(rrec, kTinest);
        }
        double s = 1.0, prod = 1.0;
#pragma unroll
        for (int i = 0; i < kEt; ++i)
            if (i < ns - 1) {
                prod = prod * r[i];
                s = s + prod;
            }
        return 1.0 / s;
    }
    __device__ __forceinline__ double element_sum(double v) const {
        double t = 0.0;
        for (int e = 0; e < m->nel; ++e) t = t + __shfl_sync(kFull, v, e);
        return t;
    }
    // species_metal_sums (species_mod.f90:566-614)
    __device__ void sums(double nH, double ne, double nHI, double nHII, double& nem, double& rin, double& rout) const {
        double pn = 0.0, pi = 0.0, po = 0.0;
        if (lane < m->nel) {
            double r[kEt];
            double fr = chain(ne, nHI, nHII, r);
            const double nX = abund * nH;
            if (ns > 1) pi = cxi[0] * nX * fr;
#pragma unroll
            for (int i = 2; i <= kMaxSt; ++i)
                if (i <= ns) {
                    fr = fr * r[i - 2];
                    pn = pn + abund * nH * fr * (double)(i - 1);
                    po = po + cxr[i - 2] * nX * fr;
                    if (i < ns) pi = pi + cxi[i - 1] * nX * fr;
                }
        }
        nem = element_sum(pn);
        rin = element_sum(pi);
        rout = element_sum(po);
    }
    // species_stage_cache_refresh (species_mod.f90:247-261): the element
    // lanes write their transitions' opacity weights
    template <typename R>
    __device__ void opacity_fill(long long l, double nH, double ne, double xHI, double colscale) const {
        if (lane >= m->nel) return;
        R* o = static_cast<R*>(m->opac) + l * m->ntrp;
        double r[kEt];
        double fr = chain(ne, nH * xHI, nH * (1.0 - xHI), r);
#pragma unroll
        for (int it = 1; it <= kEt; ++it)
            if (it <= ns - 1) {
                if (it > 1) fr = fr * r[it - 2];
                o[m->tr[tr0 + it - 1].flat] = (R)(nH * (abund * fr) * colscale);
            }
    }
    // the metal terms of net_rate (thermal_mod.f90:53-71), as metal_thermal
    __device__ MetalThermalTerms thermal(const ThermalDev& td, double T, double nH, double ne, double nHI,
                                         double nHII) const {
        const double A_CII = 2.321e-6, A_OI = 8.865e-5;
        const double rsT = 1.0 / sqrt(T);
        double lam[kStSlots];
#pragma unroll
        for (int q = 0; q < kStSlots; ++q) {
            const int sidx = lane + 32 * q;
            lam[q] = 0.0;
            if (sidx < m->nst) {
                const MetalStage& st = m->st[sidx];
                if (st.has_cool) {
                    double fit = 0.0;
                    for (int k = 0; k < st.nterm; ++k) fit = fit + st.A[k] * exp(-st.Ti[k] / T);
                    fit = fit * rsT;
                    lam[q] = st.table >= 0 ? nl_apply(m->lamref + (size_t)st.table * kNlNT,
                                                      m->Ssup + (size_t)st.table * kNlNT * kNlNNE,
                                                      m->lnL + (size_t)st.table * kNlNT * kNlNNE,
                                                      nl_at(td.tinv, T, ne), fit)
                                           : fit;
                }
            }
        }
        double lm[kMaxSt];
#pragma unroll
        for (int i = 0; i < kMaxSt; ++i) lm[i] = lane_fetch(lam, i < ns ? st0 + i : 0);
        double pc = 0.0, ph = 0.0, pf = 0.0, pq = 0.0;
        if (lane < m->nel) {
            double g[4];
            for (int z = 1; z <= 4; ++z) g[z - 1] = gbar_ff(td.gff, T, z);
            double r[kEt], frac[kMaxSt];
            frac[0] = chain(ne, nHI, nHII, r);
#pragma unroll
            for (int i = 1; i < kMaxSt; ++i) frac[i] = i < ns ? frac[i - 1] * r[i - 1] : 0.0;
            const double nel = abund * nH;
#pragma unroll
            for (int i = 0; i < kMaxSt; ++i)
                if (i < ns && ((coolmask >> i) & 1)) pc = pc + ne * nel * frac[i] * lm[i];
            if (kind == 1 && ns >= 2) {   // [C II] 158 um, H impact
                const double nion = abund * nH * frac[1];
                const double qul = 7.6e-10 * pow(T / 100.0, 0.14);
                const double qlu = 2.0 * qul * exp(-91.25 / T);
                ph = nion * nHI * qlu * (91.25 * kKboltz) / (1.0 + nHI * (qul + qlu) / A_CII);
            } else if (kind == 2) {       // [O I] 63 um
                const double nion = abund * nH * frac[0];
                const double qul = 9.2e-11 * pow(T / 100.0, 0.67);
                const double qlu = 0.6 * qul * exp(-227.7 / T);
                ph = nion * nHI * qlu * (227.7 * kKboltz) / (1.0 + nHI * (qul + qlu) / A_OI);
            }
#pragma unroll
            for (int j = 2; j <= kMaxSt; ++j)
                if (j <= ns) {
                    const int zion = j - 1;
                    pf = pf + abund * frac[j - 1] * (double)(zion * zion) * g[min(zion, 4) - 1];
                }
#pragma unroll
            for (int i = 1; i <= kEt; ++i)
                if (i <= ns - 1) pq = pq + abund * nH * frac[i - 1] * eheat[i - 1];
        }
        MetalThermalTerms o;
        o.cool = element_sum(pc);
        o.cool_H = element_sum(ph);
        o.freefree = 1.42554e-27 * sqrt(T) * ne * nH * element_sum(pf);
        o.heat = element_sum(pq);
        return o;
    }
};

__device__ __forceinline__ MetalThermalTerms thermal_terms(const ThermalDev& td, const WarpCascade& cas, long long,
                                                         double T, double nH, double ne, double nHI, double nHII) {
    return cas.thermal(td, T, nH, ne, nHI, nHII);
}

// net_rate (thermal_mod.f90:38-115).  With metals the (leaf, T) cache mc is
// prepared here at T and left for the caller.
template <class Cas>
__device__ double net_rate(const ThArgs& a, long long il, double T, double nH, double& xHI, double& xHeI,
                           double& xHeII, double& ne, int* passes, Cas& mc, int* nsum) {
    const BalArgs& b = a.b;
    const long long n = b.nleaf;
    const Coef k = coef_at_call(b.rs, b.caseA, T);
    if (b.fast) {
        if (b.m.ntr > 0) mc.prepare(il, T);
        *passes += solve_cell_fast(k, b.yHe, b.rates[il], b.rates[n + il], b.rates[2 * n + il], nH, xHI, xHeI, xHeII,
                                   ne, b.m.ntr > 0, mc, b.metal_ne, b.two_way, nsum, b.nemax);
    } else if (b.m.ntr > 0) {
        mc.prepare(il, T);
        *passes += solve_cell_metal(k, b.yHe, b.rates[il], b.rates[n + il], b.rates[2 * n + il], nH, xHI, xHeI, xHeII,
                                    ne, mc, b.metal_ne, b.two_way, nsum);
    } else {
        *passes += solve_cell(k, b.yHe, b.rates[il], b.rates[n + il], b.rates[2 * n + il], nH, xHI, xHeI, xHeII, ne);
    }
    const double heat = nH * (xHI * b.rates[3 * n + il] + b.yHe * (xHeI * b.rates[4 * n + il] + xHeII * b.rates[5 * n + il]));
    double net = heat - cooling_total(a.td, b.rs, b.caseA, b.yHe, T, nH, ne, xHI, xHeI, xHeII);
    if (b.m.ntr > 0) {
        const MetalThermalTerms mt = thermal_terms(a.td, mc, il, T, nH, ne, nH * xHI, nH * (1.0 - xHI));
        net = net - mt.cool;
        net = net - mt.cool_H;
        if (b.metal_ff) net = net - mt.freefree;
        if (b.metal_heat) net = net + mt.heat;
    }
    return net;
}

// The temperature search of the bracketed thermal solve, one leaf, driven
// by its caller one evaluation at a time: begin() at the warm start, then
// feed() the net heating at each requested temperature t until ph == 9; tr
// is the solved T_e, always the last temperature evaluated (so the cell
// state the caller holds is the one solved at it).
//
// net(T) is bracketed from the warm start by geometric steps in ln T (the
// first by fac0, each later one squaring the factor), stopping at te_min
// with net <= 0 (cooling wins) or at te_max with net >= 0 (heating wins) as
// the reference's bisection pins those leaves.  The sign change is then
// closed by Anderson-Bjorck false position in ln T: the new point replaces
// the newest end; when it keeps that end's sign the far end is retained and
// its value scaled by 1 - f_new / f_newest (by 1/2 when that is not
// positive), which moves the next point past the root.  A secant point
// within half the tolerance of the newest end is moved half the tolerance
// past the root estimate towards the far end, so one more sign change closes
// the bracket; a bracket that has not halved in three points is bisected.
// Done when the bracket is below 1e-5 in ln T (the reference's bisection
// stops at thi/tlo - 1 < 1e-5), at most 80 points.
//
// gate > 0 (the learned warm start): the warm start is accepted as the root
// after its one evaluation when |net| <= gate x (heating + cooling) there.
struct TRoot {
    int ph, s, it, stall;   // ph: 0 warm start, 1 bracketing, 2 false position, 9 done
    double ta, fa, tb, fb, fac, x1, f1, x2, f2, wref, t, tr, gate;
    bool accepted;
    __device__ __forceinline__ void begin(double Tw, double lo, double hi, double fac0 = 1.05, double g = 0.0) {
        ph = 0; s = 0; it = 0; stall = 0;
        ta = fmin(fmax(Tw, lo), hi);
        fa = 0.0; tb = ta; fb = 0.0; fac = fac0;
        x1 = x2 = f1 = f2 = wref = 0.0;
        t = ta; tr = ta;
        gate = g;
        accepted = false;
    }
    __device__ __forceinline__ void feed(double f, double lo_lim, double hi_lim, double scale = 0.0) {
        constexpr double kTol = 1.0e-5;
        bool to_fp = false;
        if (ph == 0) {
            fa = f;
            if (fa == 0.0 || (ta <= lo_lim && fa < 0.0) || (ta >= hi_lim && fa > 0.0)) {
                tr = ta;
                ph = 9;
            } else if (gate > 0.0 && fabs(fa) <= gate * scale) {
                tr = ta;
                ph = 9;
                accepted = true;
            } else {
                ph = 1;
                s = 0;
            }
        } else if (ph == 1) {
            fb = f;
            ++s;
            if (fb == 0.0) {
                tr = tb;
                ph = 9;
            } else if ((fb > 0.0) != (fa > 0.0)) {
                to_fp = true;
            } else if (tb >= hi_lim || tb <= lo_lim) {
                tr = tb;
                ph = 9;
            } else {
                ta = tb;
                fa = fb;
                fac = fac * fac;
                if (s >= 40) to_fp = true;
            }
        } else {   // ph == 2: f at t
            ++it;
            tr = t;
            if (f == 0.0) {
                ph = 9;
            } else {
                if ((f > 0.0) != (f2 > 0.0)) {
                    x1 = x2;
                    f1 = f2;
                } else {
                    const double m = 1.0 - f / f2;
                    f1 = f1 * (m > 0.0 ? m : 0.5);
                }
                x2 = log(t);
                f2 = f;
            }
        }
        if (to_fp) {
            x1 = log(ta);
            f1 = fa;
            x2 = log(tb);
            f2 = fb;
            wref = fabs(x2 - x1);
            tr = tb;
            it = 0;
            stall = 0;
            ph = 2;
        }
        if (ph == 1) {
            tb = fa > 0.0 ? fmin(ta * fac, hi_lim) : fmax(ta / fac, lo_lim);
            t = tb;
        } else if (ph == 2) {
            const double w = fabs(x2 - x1);
            if (w < kTol || it >= 80) {
                ph = 9;
            } else {
                if (w <= 0.5 * wref) {
                    wref = w;
                    stall = 0;
                } else {
                    ++stall;
                }
                double x3 = (x1 * f2 - x2 * f1) / (f2 - f1);
                if (fabs(x3 - x2) < 0.5 * kTol) x3 = x3 + copysign(0.5 * kTol, x1 - x2);
                if (stall >= 3 || !(x3 > fmin(x1, x2) && x3 < fmax(x1, x2))) {
                    x3 = 0.5 * (x1 + x2);
                    stall = 0;
                    wref = 0.5 * w;
                }
                t = exp(x3);
            }
        }
    }
};

// The bracketed T_e solve (solver_bracketed): the root of net(T) that the
// reference's bisection on [te_min, te_max] converges to (thermal_mod.f90:
// 159-180), found from a warm start T_w by the search of TRoot.  The cell
// state left behind is the one solved at the returned T_e.
template <class Cas>
__device__ double thermal_bracketed(const ThArgs& a, long long il, double nH, double& xHI, double& xHeI, double& xHeII,
                                    double& ne, int* passes, Cas& mc, int* nsum, int* nev, double Tw) {
    TRoot r;
    r.begin(Tw, a.te_min, a.te_max, a.tfac0);
    while (r.ph != 9) {
        const double f = net_rate(a, il, r.t, nH, xHI, xHeI, xHeII, ne, passes, mc, nsum);
        ++*nev;
        r.feed(f, a.te_min, a.te_max);
    }
    return r.tr;
}

// ---- the bracketed solves in warp lockstep -----------------------------------
// With one leaf per thread, the leaves of a warp need different numbers of
// root-finding steps, and a warp whose lanes sit in different loops runs the
// expensive evaluations (rate cache, cascade sums, cooling) one lane group
// at a time, reading the per-thread caches uncoalesced.  Here every root
// search is a loop whose trip count is uniform over the warp (__any_sync on
// the lanes still searching): each trip, every searching lane makes one
// evaluation at its own point, the evaluations of all lanes at the same
// program point, and then updates its own search state.  Each lane's
// sequence of points and results is that of the bracketed solves above
// (hydrogen_neutral_fraction_warm, solve_cell_fast, thermal_bracketed).
// Every function here is entered by all 32 lanes; `act` marks the lanes
// whose leaf takes part.

// The H root with charge exchange (hydrogen_neutral_fraction_warm, falling
// back to hydrogen_neutral_fraction's Illinois iteration).
__device__ __noinline__ double h_root_ls(const SerialCascade& mc, bool act, double nH, double ne, double A, double B,
                                         double xg, int* nsum, double* nem_x) {
    // ph: 0 substitution, 1-2 Illinois end points x = 0, 1, 3 Illinois steps,
    // 4 the sums at the Illinois root, 5 done
    int ph = act ? 0 : 5, k = 0, kk = 0;
    double x = fmin(fmax(xg, 0.0), 1.0), prev = 1.0e300;
    double xa = 0.0, xb = 1.0, Ra = 0.0, Rb = 0.0, scale = 0.0, nem = 0.0;
    while (__any_sync(kFull, ph != 5)) {
        if (ph == 5) continue;
        const double xe = ph == 1 ? 0.0 : ph == 2 ? 1.0 : x;
        double em, rin, rout;
        mc.sums(nH, ne, nH * xe, nH * (1.0 - xe), em, rin, rout);
        ++*nsum;
        if (ph == 0) {
            const double Rx = x * (B + rin + rout) - (A + rin);
            const double sc = A + B + fabs(A + rin) + fabs(B + rout);
            const double xn = fmin(fmax((A + rin) / (B + rin + rout), 0.0), 1.0);
            const int v = h_subst_verdict(x, xn, Rx, sc, prev);
            if (v == 1) {
                nem = em;
                ph = 5;
            } else if (v == 2 || ++k >= 8) {
                ph = 1;
            } else {
                prev = fabs(Rx);
                x = xn;
            }
        } else if (ph == 1) {
            Ra = -(A + rin);
            ph = 2;
        } else if (ph == 2) {
            Rb = B + rout;
            scale = A + B + fabs(Ra) + fabs(Rb);
            x = xb;
            kk = 0;
            ph = 3;
        } else if (ph == 3) {
            const double Rx = x * (B + rin + rout) - (A + rin);
            if (fabs(Rx) <= 1.0e-15 * scale || fabs(xb - xa) <= 1.0e-15) {
                ph = 4;
            } else {
                if (Rx * Rb < 0.0) {
                    xa = xb;
                    Ra = Rb;
                } else {
                    Ra = 0.5 * Ra;
                }
                xb = x;
                Rb = Rx;
            }
        } else {   // ph == 4
            nem = em;
            ph = 5;
        }
        if (ph == 3) {   // the next Illinois point (hydrogen_neutral_fraction's loop head)
            if (++kk > 80 || Rb == Ra) {
                ph = 4;
            } else {
                x = xb - Rb * (xb - xa) / (Rb - Ra);
                x = fmin(fmax(x, fmin(xa, xb)), fmax(xa, xb));
            }
        }
    }
    *nem_x = nem;
    return x;
}

__device__ __forceinline__ double cell_electrons_ls(const Coef& k, double yHe, double gH, double gHe1, double gHe2,
                                                    double nH, double ne, bool act, const SerialCascade& mc,
                                                    int with_ne, int with_cx, int* nsum, CellState& o, double xg) {
    double nem_x = 0.0;
    if (with_cx) {
        o.x = h_root_ls(mc, act, nH, ne, k.aH * ne, gH + (k.cH + k.aH) * ne, xg, nsum, &nem_x);
    } else if (act) {
        const double denH = gH + (k.cH + k.aH) * ne;
        o.x = denH > 0.0 ? (k.aH * ne) / denH : 1.0;
    }
    if (!act) return 0.0;
    const double r1 = fmin((gHe1 + k.cHe1 * ne) / (k.aHe2 * ne), 1.0e150);
    const double r2 = fmin((gHe2 + k.cHe2 * ne) / (k.aHe3 * ne), 1.0e150);
    o.h1 = 1.0 / (1.0 + r1 + r1 * r2);
    o.h2 = o.h1 * r1;
    const double h3 = o.h2 * r2;
    double nen = nH * ((1.0 - o.x) + yHe * (o.h2 + 2.0 * h3));
    if (with_ne) {
        if (!with_cx) {
            double rin, rout;
            mc.sums(nH, ne, nH * o.x, nH * (1.0 - o.x), nem_x, rin, rout);
            ++*nsum;
        }
        nen = nen + nem_x;
    }
    return nen;
}

// solve_cell_fast with metals as a per-lane state machine.
__device__ __noinline__ int solve_cell_ls(const Coef& k, double yHe, double gH, double gHe1, double gHe2, double nH,
                                          double& xHI, double& xHeI, double& xHeII, double& ne, bool act,
                                          const SerialCascade& mc, int with_ne, int with_cx, int* nsum, double nemax) {
    const double floor = 1.0e-12 * nH, top = nemax * nH;
    double a = 0.0, fa = 0.0, b = 0.0, fb = 0.0, c = 0.0, fac = 4.0, la = 0.0, lb = 0.0;
    int ph = act ? 0 : 9, nev = 0, side = 0, it = 0;   // 0 first point, 1 search, 2 false position, 9 done
    CellState ea = {xHI, xHeI, xHeII}, eb = ea, ec = ea;
    if (act) {
        const double xHeIII = fmax(0.0, 1.0 - xHeI - xHeII);
        a = ne > floor ? ne : fmax(nH * ((1.0 - xHI) + yHe * (xHeII + 2.0 * xHeIII)), floor);
        a = fmin(a, top);
        c = a;
    }
    while (__any_sync(kFull, ph != 9)) {
        const bool ev = ph != 9;
        const double fc = cell_electrons_ls(k, yHe, gH, gHe1, gHe2, nH, c, ev, mc, with_ne, with_cx, nsum, ec, ec.x) - c;
        if (!ev) continue;
        ++nev;
        bool to_fp = false;
        if (ph == 0) {
            fa = fc; ea = ec; b = a; fb = fa; eb = ea;
            if (fabs(fa) <= 2.0e-10 * a) {
                ph = 9;
            } else {
                c = fa > 0.0 ? fmin(a + fa, top) : fmax(a + fa, floor);
                if (!(c > 0.0)) c = floor;
                ph = 1;
            }
        } else if (ph == 1) {
            b = c; fb = fc; eb = ec;
            if (fabs(fc) <= 2.0e-10 * c || fc == 0.0) {
                ph = 9;
            } else if ((fc > 0.0) != (fa > 0.0)) {
                to_fp = true;
            } else if (c >= top || c <= floor) {
                ph = 9;
            } else {
                const double lA = log(a), lC = log(c);
                double ld = lC - fc * (lC - lA) / (fc - fa);
                const bool ahead = fc > 0.0 ? ld > lC : ld < lC;
                const double lim = log(fac);
                if (!(fabs(fc) < fabs(fa)) || !ahead || !(fabs(ld - lC) <= lim)) ld = fc > 0.0 ? lC + lim : lC - lim;
                a = c; fa = fc; ea = ec;
                c = fc > 0.0 ? fmin(exp(ld), top) : fmax(exp(ld), floor);
                fac = fac * fac;
                if (nev >= 60) to_fp = true;
            }
        } else {   // ph == 2: Anderson-Bjorck step at c
            b = c;
            eb = ec;
            ++it;
            const double lc = log(c);
            if (fabs(fc) <= 2.0e-10 * c || fc == 0.0) {
                ph = 9;
            } else if ((fc > 0.0) == (fb > 0.0)) {
                if (side == -1) {
                    const double m = 1.0 - fc / fb;
                    fa = fa * (m > 0.0 ? m : 0.5);
                }
                lb = lc; fb = fc; side = -1;
            } else {
                if (side == +1) {
                    const double m = 1.0 - fc / fa;
                    fb = fb * (m > 0.0 ? m : 0.5);
                }
                la = lc; fa = fc; side = +1;
            }
        }
        if (to_fp) {
            la = log(a);
            lb = log(b);
            side = 0;
            it = 0;
            ph = 2;
        }
        if (ph == 2) {   // the next false-position point, or the end of the search
            const double width = fabs(lb - la);
            if (width <= 1.0e-13 || it >= 100 || nev >= 160) {
                ph = 9;
            } else {
                double lc = (la * fb - lb * fa) / (fb - fa);
                if (!(fabs(lc - la) > 1.0e-3 * width && fabs(lc - lb) > 1.0e-3 * width)) lc = 0.5 * (la + lb);
                c = exp(lc);
            }
        }
    }
    if (act) {
        ne = b;
        xHI = eb.x;
        xHeI = eb.h1;
        xHeII = eb.h2;
    }
    return nev;
}

__device__ __noinline__ double net_rate_ls(const ThArgs& a, long long il, bool act, double T, double nH, double& xHI,
                                           double& xHeI, double& xHeII, double& ne, int* passes, SerialCascade& mc,
                                           int* nsum) {
    const BalArgs& b = a.b;
    const long long n = b.nleaf;
    Coef k = {};
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    if (act) {
        k = coef_at_call(b.rs, b.caseA, T);
        mc.prepare(il, T);
        g0 = b.rates[il]; g1 = b.rates[n + il]; g2 = b.rates[2 * n + il];
    }
    *passes += solve_cell_ls(k, b.yHe, g0, g1, g2, nH, xHI, xHeI, xHeII, ne, act, mc, b.metal_ne, b.two_way, nsum,
                             b.nemax);
    if (!act) return 0.0;
    const double heat = nH * (xHI * b.rates[3 * n + il] + b.yHe * (xHeI * b.rates[4 * n + il] + xHeII * b.rates[5 * n + il]));
    double net = heat - cooling_total(a.td, b.rs, b.caseA, b.yHe, T, nH, ne, xHI, xHeI, xHeII);
    const MetalThermalTerms mt = thermal_terms(a.td, mc, il, T, nH, ne, nH * xHI, nH * (1.0 - xHI));
    net = net - mt.cool;
    net = net - mt.cool_H;
    if (b.metal_ff) net = net - mt.freefree;
    if (b.metal_heat) net = net + mt.heat;
    return net;
}

// thermal_bracketed as a per-lane state machine.
__device__ __noinline__ double thermal_ls(const ThArgs& a, long long il, bool act, double nH, double& xHI,
                                          double& xHeI, double& xHeII, double& ne, int* passes, SerialCascade& mc,
                                          int* nsum, int* nev, double Tw) {
    TRoot r;
    r.begin(Tw, a.te_min, a.te_max, a.tfac0);
    if (!act) r.ph = 9;
    while (__any_sync(kFull, r.ph != 9)) {
        const bool ev = r.ph != 9;
        const double f = net_rate_ls(a, il, ev, r.t, nH, xHI, xHeI, xHeII, ne, passes, mc, nsum);
        if (!ev) continue;
        ++*nev;
        r.feed(f, a.te_min, a.te_max);
    }
    return r.tr;
}

// gas_thermal_update (thermal_mod.f90:124-249): bisection on log T in
// [te_min, te_max] (at most 60 halvings, stop at thi/tlo - 1 < 1e-5), the
// ionisation re-solved at every trial temperature.
__global__ void __launch_bounds__(kBThreads) k_thermal(const ThArgs a) {
    __shared__ double sh[6][kBThreads];
    const BalArgs& b = a.b;
    double mdx = 0.0, mdt = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
    unsigned long long solved = 0, caps = 0, tpass = 0, tsums = 0, nevals = 0;
    for (long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x; il < b.nleaf;
         il += (long long)gridDim.x * blockDim.x) {
        const double nH = b.nH[il];
        const double x0 = b.xHI[il], h10 = b.xHeI[il], h20 = b.xHeII[il], T0 = b.Te[il];
        if (nH <= 0.0) {
            b.ne[il] = 0.0;
            write_columns(b.col, il, b.nabs, b.fp32, nH, b.yHe, x0, h10, h20, b.colscale, b.rhokap ? b.rhokap[il] : 0.0);
            continue;
        }
        double xHI = x0, xHeI = h10, xHeII = h20, ne = 0.0;
        int passes = 0, nsum = 0, nev = 0, last = 0;
        double te;
        SerialCascade mc;
        mc.m = &b.m;
        if (b.fast) {
            ne = b.ne[il];
            te = thermal_bracketed(a, il, nH, xHI, xHeI, xHeII, ne, &passes, mc, &nsum, &nev,
                                   a.Twarm ? a.Twarm[il] : T0);
        } else {
            double tlo = a.te_min, thi = a.te_max;
            nev = 3;
            const double net_lo = net_rate(a, il, tlo, nH, xHI, xHeI, xHeII, ne, &passes, mc, &nsum);
            const double net_hi = net_rate(a, il, thi, nH, xHI, xHeI, xHeII, ne, &passes, mc, &nsum);
            if (net_lo <= 0.0) {
                te = tlo;
            } else if (net_hi >= 0.0) {
                te = thi;
            } else {
                for (int it = 1; it <= 60; ++it) {
                    const double tmid = sqrt(tlo * thi);
                    const double nm = net_rate(a, il, tmid, nH, xHI, xHeI, xHeII, ne, &passes, mc, &nsum);
                    ++nev;
                    if (nm > 0.0) tlo = tmid; else thi = tmid;
                    if (thi / tlo - 1.0 < 1.0e-5) break;
                }
                te = sqrt(tlo * thi);
            }
            net_rate(a, il, te, nH, xHI, xHeI, xHeII, ne, &last, mc, &nsum);
            if (last > 200) ++caps;
        }
        ++solved;
        tpass += (unsigned long long)(passes + last);
        tsums += (unsigned long long)nsum;
        nevals += (unsigned long long)nev;
        const double w = b.relax;
        const double xn = (1.0 - w) * x0 + w * xHI;
        const double h1n = (1.0 - w) * h10 + w * xHeI;
        const double h2n = (1.0 - w) * h20 + w * xHeII;
        const double h3n = fmax(0.0, 1.0 - h1n - h2n);
        double nen = nH * ((1.0 - xn) + b.yHe * (h2n + 2.0 * h3n));
        if (b.m.ntr > 0) {
            // written state at te (thermal_mod.f90:191-203); mc is at te from
            // the final net_rate, which is also the stage cache's temperature
            if (b.metal_ne) nen = charge_neutrality_ne(mc, nH, nen, xn, ne);
            if (b.fp32) mc.opacity_fill<float>(il, nH, nen, xn, b.colscale);
            else mc.opacity_fill<double>(il, nH, nen, xn, b.colscale);
        }
        b.xHI[il] = xn;
        b.xHeI[il] = h1n;
        b.xHeII[il] = h2n;
        b.ne[il] = nen;
        b.Te[il] = te;
        write_columns(b.col, il, b.nabs, b.fp32, nH, b.yHe, xn, h1n, h2n, b.colscale, b.rhokap ? b.rhokap[il] : 0.0);
        const double dx = fabs(xn - x0);
        mdx = fmax(mdx, dx);
        mdt = fmax(mdt, fabs(te - T0) / T0);
        const double vol = leaf_vol(b, il);
        s1 = s1 + vol * dx;
        s2 = s2 + vol * (1.0 - xn);
        s3 = s3 + vol * nen * fabs(te - T0);
        s4 = s4 + vol * nen * te;
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
        tpass += __shfl_down_sync(0xffffffffu, tpass, o);
        tsums += __shfl_down_sync(0xffffffffu, tsums, o);
        nevals += __shfl_down_sync(0xffffffffu, nevals, o);
    }
    if ((t & 31) == 0) {
        if (solved) atomicAdd(b.counters + 0, solved);
        if (caps) atomicAdd(b.counters + 1, caps);
        if (tpass) atomicAdd(b.counters + 2, tpass);
        if (tsums) atomicAdd(b.counters + 3, tsums);
        if (nevals) atomicAdd(b.counters + 4, nevals);
    }
}

__global__ void k_iota(int* v, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// charge_neutrality_ne in warp lockstep.
__device__ __noinline__ double neutrality_ls(const SerialCascade& mc, bool act, double nH, double ne_HHe, double xHI,
                                             double ne_seed) {
    const double nHI = nH * xHI, nHII = nH * (1.0 - xHI);
    double ne = fmax(ne_seed, 1.0e-12 * nH);
    int it = 0;
    bool run = act;
    while (__any_sync(kFull, run)) {
        if (!run) continue;
        const double ne_old = ne;
        double nem, rin, rout;
        mc.sums(nH, ne_old, nHI, nHII, nem, rin, rout);
        ne = ne_HHe + nem;
        ne = fmax(0.5 * (ne + ne_old), 1.0e-12 * nH);
        if (fabs(ne - ne_old) <= 1.0e-10 * ne || ++it >= 200) run = false;
    }
    return ne;
}

// gas_thermal_update with metals and the bracketed solve, one leaf per
// thread in warp lockstep (thermal_ls).  Persistent warps claim chunks of 32
// consecutive leaves of the work order (the most work first) from a global
// counter, so every lane of a warp makes the same number of trips and a warp
// that finishes early takes more leaves instead of idling.
// The per-lane sums a thermal kernel reports (thermal_mod.f90:223-224 and the
// solver counters).
struct ThermalAcc {
    double mdx = 0.0, mdt = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
    unsigned long long solved = 0, tpass = 0, tsums = 0, nevals = 0;
    unsigned long long accepted = 0;   // learned warm starts accepted by the residual gate
};

// One warp's 32 leaves at positions base .. base+31 of a's order, in lockstep.
__device__ __forceinline__ void thermal_chunk_ls(const ThArgs& a, long long base, int lane, ThermalAcc& acc) {
    const BalArgs& b = a.b;
    const long long i0 = base + lane;
    const bool valid = i0 < b.nleaf;
    const long long ip = valid ? i0 : b.nleaf - 1;
    const long long il = a.order ? (long long)a.order[b.nleaf - 1 - ip] : ip;
    const double nH = b.nH[il];
    const double x0 = b.xHI[il], h10 = b.xHeI[il], h20 = b.xHeII[il], T0 = b.Te[il];
    const bool act = valid && nH > 0.0;
    if (valid && !act) {
        b.ne[il] = 0.0;
        write_columns(b.col, il, b.nabs, b.fp32, nH, b.yHe, x0, h10, h20, b.colscale,
                      b.rhokap ? b.rhokap[il] : 0.0);
        if (a.work) a.work[il] = 0u;
    }
    double xHI = x0, xHeI = h10, xHeII = h20, ne = b.ne[il];
    int passes = 0, nsum = 0, nev = 0;
    SerialCascade mc;
    mc.m = &b.m;
    const double te = thermal_ls(a, il, act, nH, xHI, xHeI, xHeII, ne, &passes, mc, &nsum, &nev,
                                 a.Twarm ? a.Twarm[il] : T0);
    const double w = b.relax;
    const double xn = (1.0 - w) * x0 + w * xHI;
    const double h1n = (1.0 - w) * h10 + w * xHeI;
    const double h2n = (1.0 - w) * h20 + w * xHeII;
    const double h3n = fmax(0.0, 1.0 - h1n - h2n);
    double nen = nH * ((1.0 - xn) + b.yHe * (h2n + 2.0 * h3n));
    // written state at te (thermal_mod.f90:191-203); the cache is at te from
    // the final net_rate
    if (b.metal_ne) nen = neutrality_ls(mc, act, nH, nen, xn, ne);
    if (!act) return;
    if (b.fp32) mc.opacity_fill<float>(il, nH, nen, xn, b.colscale);
    else mc.opacity_fill<double>(il, nH, nen, xn, b.colscale);
    ++acc.solved;
    acc.tpass += (unsigned long long)passes;
    acc.tsums += (unsigned long long)nsum;
    acc.nevals += (unsigned long long)nev;
    if (a.work) a.work[il] = (unsigned)min(nsum, 65535);
    b.xHI[il] = xn;
    b.xHeI[il] = h1n;
    b.xHeII[il] = h2n;
    b.ne[il] = nen;
    b.Te[il] = te;
    write_columns(b.col, il, b.nabs, b.fp32, nH, b.yHe, xn, h1n, h2n, b.colscale, b.rhokap ? b.rhokap[il] : 0.0);
    const double dx = fabs(xn - x0);
    acc.mdx = fmax(acc.mdx, dx);
    acc.mdt = fmax(acc.mdt, fabs(te - T0) / T0);
    const double vol = leaf_vol(b, il);
    acc.s1 = acc.s1 + vol * dx;
    acc.s2 = acc.s2 + vol * (1.0 - xn);
    acc.s3 = acc.s3 + vol * nen * fabs(te - T0);
    acc.s4 = acc.s4 + vol * nen * te;
}

__global__ void __launch_bounds__(kBThreads) k_thermal_ls(const ThArgs a) {
    __shared__ double sh[6][kBThreads];
    const BalArgs& b = a.b;
    ThermalAcc acc;
    const int lane = threadIdx.x & 31;
    const long long nwarp = (long long)gridDim.x * (blockDim.x >> 5);
    long long chunk = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    for (;;) {
        const long long base = chunk * 32;
        if (base >= b.nleaf) break;
        {   // the next chunk
            unsigned long long c = 0;
            if (lane == 0) c = atomicAdd(a.next, 1ull);
            chunk = nwarp + (long long)__shfl_sync(kFull, c, 0);
        }
        thermal_chunk_ls(a, base, lane, acc);
    }
    const int t = threadIdx.x;
    sh[0][t] = acc.mdx; sh[1][t] = acc.mdt; sh[2][t] = acc.s1; sh[3][t] = acc.s2; sh[4][t] = acc.s3; sh[5][t] = acc.s4;
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
    unsigned long long solved = acc.solved, tpass = acc.tpass, tsums = acc.tsums, nevals = acc.nevals;
    for (int o = 16; o > 0; o >>= 1) {
        solved += __shfl_down_sync(kFull, solved, o);
        tpass += __shfl_down_sync(kFull, tpass, o);
        tsums += __shfl_down_sync(kFull, tsums, o);
        nevals += __shfl_down_sync(kFull, nevals, o);
    }
    if ((t & 31) == 0) {
        if (solved) atomicAdd(b.counters + 0, solved);
        if (tpass) atomicAdd(b.counters + 2, tpass);
        if (tsums) atomicAdd(b.counters + 3, tsums);
        if (nevals) atomicAdd(b.counters + 4, nevals);
    }
}

// A warp's sums into its nebula's first partial slot and counters (the
// values are non-negative, so their bit patterns order as the numbers).
__device__ __forceinline__ void thermal_acc_flush(const BalArgs& b, ThermalAcc& acc) {
    double v[6] = {acc.mdx, acc.mdt, acc.s1, acc.s2, acc.s3, acc.s4};
    unsigned long long c[5] = {acc.solved, acc.tpass, acc.tsums, acc.nevals, acc.accepted};
    for (int o = 16; o > 0; o >>= 1) {
        v[0] = fmax(v[0], __shfl_down_sync(kFull, v[0], o));
        v[1] = fmax(v[1], __shfl_down_sync(kFull, v[1], o));
        for (int k = 2; k < 6; ++k) v[k] += __shfl_down_sync(kFull, v[k], o);
        for (int k = 0; k < 5; ++k) c[k] += __shfl_down_sync(kFull, c[k], o);
    }
    if ((threadIdx.x & 31) == 0) {
        unsigned long long* pm = reinterpret_cast<unsigned long long*>(b.partial);
        atomicMax(pm + 0, (unsigned long long)__double_as_longlong(v[0]));
        atomicMax(pm + 1, (unsigned long long)__double_as_longlong(v[1]));
        for (int k = 2; k < 6; ++k) atomicAdd(b.partial + k, v[k]);
        if (c[0]) atomicAdd(b.counters + 0, c[0]);
        if (c[1]) atomicAdd(b.counters + 2, c[1]);
        if (c[2]) atomicAdd(b.counters + 3, c[2]);
        if (c[3]) atomicAdd(b.counters + 4, c[3]);
        if (c[4]) atomicAdd(b.counters + 5, c[4]);
    }
    acc = ThermalAcc();
}

#include "thermal_lane.cuh"

// The lockstep thermal solve of many nebulae in one persistent launch: the
// 32-leaf chunks of all nebulae are numbered consecutively (chunk_off: the
// first chunk of each nebula, nneb + 1 entries) and claimed from one counter;
// a warp copies its nebula's arguments into shared memory and reports its
// sums to that nebula when it moves to another one or ends.
__global__ void __launch_bounds__(kBThreads) k_thermal_batch(const ThArgs* __restrict__ args, int nneb,
                                                             const long long* __restrict__ chunk_off,
                                                             unsigned long long* next) {
    __shared__ ThArgs sa[kBThreads / 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long total = chunk_off[nneb];
    const long long nwarp = (long long)gridDim.x * (blockDim.x >> 5);
    long long chunk = (long long)blockIdx.x * (blockDim.x >> 5) + wib;
    int cur = -1;
    ThermalAcc acc;
    for (;;) {
        if (chunk >= total) break;
        int k = 0;   // the nebula of this chunk
        {
            int lo = 0, hi = nneb - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (chunk_off[mid] <= chunk) lo = mid; else hi = mid - 1;
            }
            k = lo;
        }
        if (k != cur) {
            if (cur >= 0) thermal_acc_flush(sa[wib].b, acc);
            __syncwarp();
            const int nw = (int)(sizeof(ThArgs) / 4);
            const unsigned* src = reinterpret_cast<const unsigned*>(args + k);
            unsigned* dst = reinterpret_cast<unsigned*>(sa + wib);
            for (int q = lane; q < nw; q += 32) dst[q] = src[q];
            __syncwarp();
            cur = k;
        }
        const long long base = (chunk - chunk_off[k]) * 32;
        {
            unsigned long long c = 0;
            if (lane == 0) c = atomicAdd(next, 1ull);
            chunk = nwarp + (long long)__shfl_sync(kFull, c, 0);
        }
        thermal_chunk_ls(sa[wib], base, lane, acc);
    }
    if (cur >= 0) thermal_acc_flush(sa[wib].b, acc);
}

// The per-lane solve (k_thermal_lane) of many nebulae in one persistent
// launch: every warp takes the nebulae in turn, its lanes claiming leaves of
// nebula q's work order from next[q] until it is exhausted; the warp's sums
// go to nebula q before it moves on.
__global__ void __launch_bounds__(kBThreads, 1) k_thermal_lane_batch(const ThArgs* __restrict__ args, int nneb,
                                                                     unsigned long long* next) {
    extern __shared__ __align__(16) unsigned char lane_smem[];
    __shared__ ThArgs sa[kBThreads / 32];
    __shared__ LaneLayout sl[kBThreads / 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double* S = reinterpret_cast<double*>(lane_smem);
    for (int q = 0; q < nneb; ++q) {
        __syncwarp();
        const int nw = (int)(sizeof(ThArgs) / 4);
        const unsigned* src = reinterpret_cast<const unsigned*>(args + q);
        unsigned* dst = reinterpret_cast<unsigned*>(sa + wib);
        for (int k = lane; k < nw; k += 32) dst[k] = src[k];
        __syncwarp();
        if (lane == 0) lane_layout_build(sa[wib].b.m, sl[wib]);
        __syncwarp();
        LaneCache cache{S + threadIdx.x, (int)blockDim.x, &sl[wib], &sa[wib].b.m, sa[wib].b.m.el, sa[wib].b.m.nel};
        ThermalAcc acc;
        lane_solve(sa[wib], next + q, cache, acc, lane);
        thermal_acc_flush(sa[wib].b, acc);
    }
}

// ---- the bracketed thermal solve as one flat per-lane state machine ---------
// The nested lockstep loops above still make a warp wait, at every level,
// for its slowest lane (the T steps, the n_e steps within a T step, the H
// root within an n_e step).  Here each lane runs its leaf's whole solve as
// one state machine (LeafFlow) that stops only to ask for an expensive
// evaluation -- the rate cache at a new T (kReqPrepare), one cascade sum
// (kReqSums), or the net heating at the solved state (kReqFinish) -- and the
// warp serves each kind of request for all lanes that ask for it, once per
// trip.  A lane whose leaf is done takes the next leaf of the (work-sorted)
// order from a global counter.  Each lane's sequence of points and results
// is that of thermal_bracketed / solve_cell_fast /
// hydrogen_neutral_fraction_warm / charge_neutrality_ne.
enum : int { kReqNone = 0, kReqPrepare = 1, kReqSums = 2, kReqFinish = 3 };

struct LeafFlow {
    const ThArgs* A;
    int req = kReqNone;
    bool live = false;
    // the leaf
    long long pos = 0, il = 0;
    double nH = 0, x0 = 0, h10 = 0, h20 = 0, T0 = 0;
    double xHI = 0, xHeI = 0, xHeII = 0, ne = 0;
    int passes = 0, nsum = 0, nev = 0;
    // request arguments
    double q_T = 0, q_ne = 0, q_x = 0;
    // T level (thermal_bracketed)
    TRoot tsr;
    // net_rate level
    Coef k = {};
    double g0 = 0, g1 = 0, g2 = 0;
    // n_e level (solve_cell_fast)
    int eph = 0, enev = 0, eside = 0, eit = 0;
    double ea = 0, efa = 0, eb = 0, efb = 0, ec = 0, efac = 4.0, ela = 0, elb = 0;
    CellState Sa = {}, Sb = {}, Sc = {};
    // F level (cell_electrons at ec)
    int fph = 0;
    double fnem = 0;
    // H root level
    int hph = 0, hk = 0, hkk = 0;
    double hx = 0, hprev = 0, hxa = 0, hxb = 0, hRa = 0, hRb = 0, hscale = 0, hA = 0, hB = 0;
    // leaf end: n_e closure of the written state
    int nit = 0;
    double te = 0, xn = 0, h1n = 0, h2n = 0, nen_hhe = 0, nen = 0;
    bool in_neu = false;

    __device__ void start_leaf(long long p, long long leaf) {
        const BalArgs& b = A->b;
        pos = p;
        il = leaf;
        nH = b.nH[il];
        x0 = b.xHI[il]; h10 = b.xHeI[il]; h20 = b.xHeII[il]; T0 = b.Te[il];
        xHI = x0; xHeI = h10; xHeII = h20; ne = b.ne[il];
        passes = nsum = nev = 0;
        in_neu = false;
        live = true;
        // thermal_bracketed: the warm start
        tsr.begin(A->Twarm ? A->Twarm[il] : T0, A->te_min, A->te_max, A->tfac0);
        start_net(tsr.t);
    }
    __device__ void start_net(double T) {
        q_T = T;
        req = kReqPrepare;
    }
    // after the rate cache is at q_T (the warp ran prepare)
    __device__ void on_prepare() {
        const BalArgs& b = A->b;
        const long long n = b.nleaf;
        k = coef_at_call(b.rs, b.caseA, q_T);
        g0 = b.rates[il]; g1 = b.rates[n + il]; g2 = b.rates[2 * n + il];
        // solve_cell_fast: the first point
        const double floor = 1.0e-12 * nH, top = b.nemax * nH;
        const double xHeIII = fmax(0.0, 1.0 - xHeI - xHeII);
        ea = ne > floor ? ne : fmax(nH * ((1.0 - xHI) + b.yHe * (xHeII + 2.0 * xHeIII)), floor);
        ea = fmin(ea, top);
        enev = 0;
        efac = 4.0;
        Sc = {xHI, xHeI, xHeII};
        eph = 0;
        start_F(ea);
    }
    __device__ void start_F(double c) {
        ec = c;
        if (A->b.two_way) {
            hA = k.aH * c;
            hB = g0 + (k.cH + k.aH) * c;
            hx = fmin(fmax(Sc.x, 0.0), 1.0);
            hprev = 1.0e300;
            hk = 0;
            hph = 0;
            fph = 0;
            ask_sums(c, hx);
        } else {
            const double denH = g0 + (k.cH + k.aH) * c;
            Sc.x = denH > 0.0 ? (k.aH * c) / denH : 1.0;
            after_x(0.0, false);
        }
    }
    __device__ void ask_sums(double c, double x) {
        q_ne = c;
        q_x = x;
        req = kReqSums;
    }
    __device__ void on_sums(double em, double rin, double rout) {
        if (in_neu) { on_neu(em); return; }   // the closure's sums are not counted (as charge_neutrality_ne)
        ++nsum;
        if (fph == 1) { after_nem(em); return; }
        // H root (hydrogen_neutral_fraction_warm)
        if (hph == 0) {
            const double Rx = hx * (hB + rin + rout) - (hA + rin);
            const double sc = hA + hB + fabs(hA + rin) + fabs(hB + rout);
            const double xn_ = fmin(fmax((hA + rin) / (hB + rin + rout), 0.0), 1.0);
            const int v = h_subst_verdict(hx, xn_, Rx, sc, hprev);
            if (v == 1) {
                Sc.x = hx;
                after_x(em, true);
                return;
            }
            if (v == 2 || ++hk >= 8) {
                hph = 1;
                ask_sums(ec, 0.0);
                return;
            }
            hprev = fabs(Rx);
            hx = xn_;
            ask_sums(ec, hx);
            return;
        }
        if (hph == 1) {
            hRa = -(hA + rin);
            hph = 2;
            ask_sums(ec, 1.0);
            return;
        }
        if (hph == 2) {
            hRb = hB + rout;
            hscale = hA + hB + fabs(hRa) + fabs(hRb);
            hxa = 0.0;
            hxb = 1.0;
            hx = hxb;
            hkk = 0;
            hph = 3;
        } else if (hph == 3) {
            const double Rx = hx * (hB + rin + rout) - (hA + rin);
            if (fabs(Rx) <= 1.0e-15 * hscale || fabs(hxb - hxa) <= 1.0e-15) {
                hph = 4;
            } else {
                if (Rx * hRb < 0.0) {
                    hxa = hxb;
                    hRa = hRb;
                } else {
                    hRa = 0.5 * hRa;
                }
                hxb = hx;
                hRb = Rx;
            }
        } else {   // hph == 4: the sums at the Illinois root
            Sc.x = hx;
            after_x(em, true);
            return;
        }
        if (hph == 3) {
            if (++hkk > 80 || hRb == hRa) {
                hph = 4;
            } else {
                hx = hxb - hRb * (hxb - hxa) / (hRb - hRa);
                hx = fmin(fmax(hx, fmin(hxa, hxb)), fmax(hxa, hxb));
            }
        }
        ask_sums(ec, hx);
    }
    // cell_electrons after x_HI: He, then the metal electrons
    __device__ void after_x(double nem_x, bool have_nem) {
        const BalArgs& b = A->b;
        const double c = ec;
        const double r1 = fmin((g1 + k.cHe1 * c) / (k.aHe2 * c), 1.0e150);
        const double r2 = fmin((g2 + k.cHe2 * c) / (k.aHe3 * c), 1.0e150);
        Sc.h1 = 1.0 / (1.0 + r1 + r1 * r2);
        Sc.h2 = Sc.h1 * r1;
        if (b.metal_ne && !have_nem) {
            fph = 1;
            ask_sums(c, Sc.x);
            return;
        }
        after_nem(b.metal_ne ? nem_x : 0.0);
    }
    __device__ void after_nem(double nem) {
        const BalArgs& b = A->b;
        fph = 0;
        const double h3 = Sc.h2 * fmin((g2 + k.cHe2 * ec) / (k.aHe3 * ec), 1.0e150);
        double nenF = nH * ((1.0 - Sc.x) + b.yHe * (Sc.h2 + 2.0 * h3));
        if (b.metal_ne) nenF = nenF + nem;
        on_F(nenF - ec);
    }
    // solve_cell_fast after F(ec) = fc
    __device__ void on_F(double fc) {
        const BalArgs& b = A->b;
        const double floor = 1.0e-12 * nH, top = b.nemax * nH;
        ++enev;
        bool to_fp = false;
        if (eph == 0) {
            efa = fc; Sa = Sc; eb = ea; efb = efa; Sb = Sa;
            if (fabs(efa) <= 2.0e-10 * ea) {
                eph = 9;
            } else {
                double c = efa > 0.0 ? fmin(ea + efa, top) : fmax(ea + efa, floor);
                if (!(c > 0.0)) c = floor;
                ec = c;
                eph = 1;
            }
        } else if (eph == 1) {
            eb = ec; efb = fc; Sb = Sc;
            if (fabs(fc) <= 2.0e-10 * ec || fc == 0.0) {
                eph = 9;
            } else if ((fc > 0.0) != (efa > 0.0)) {
                to_fp = true;
            } else if (ec >= top || ec <= floor) {
                eph = 9;
            } else {
                const double lA = log(ea), lC = log(ec);
                double ld = lC - fc * (lC - lA) / (fc - efa);
                const bool ahead = fc > 0.0 ? ld > lC : ld < lC;
                const double lim = log(efac);
                if (!(fabs(fc) < fabs(efa)) || !ahead || !(fabs(ld - lC) <= lim)) ld = fc > 0.0 ? lC + lim : lC - lim;
                ea = ec; efa = fc; Sa = Sc;
                ec = fc > 0.0 ? fmin(exp(ld), top) : fmax(exp(ld), floor);
                efac = efac * efac;
                if (enev >= 60) to_fp = true;
            }
        } else {   // eph == 2
            eb = ec;
            Sb = Sc;
            ++eit;
            const double lc = log(ec);
            if (fabs(fc) <= 2.0e-10 * ec || fc == 0.0) {
                eph = 9;
            } else if ((fc > 0.0) == (efb > 0.0)) {
                if (eside == -1) {
                    const double m = 1.0 - fc / efb;
                    efa = efa * (m > 0.0 ? m : 0.5);
                }
                elb = lc; efb = fc; eside = -1;
            } else {
                if (eside == +1) {
                    const double m = 1.0 - fc / efa;
                    efb = efb * (m > 0.0 ? m : 0.5);
                }
                ela = lc; efa = fc; eside = +1;
            }
        }
        if (to_fp) {
            ela = log(ea);
            elb = log(eb);
            eside = 0;
            eit = 0;
            eph = 2;
        }
        if (eph == 2) {
            const double width = fabs(elb - ela);
            if (width <= 1.0e-13 || eit >= 100 || enev >= 160) {
                eph = 9;
            } else {
                double lc = (ela * efb - elb * efa) / (efb - efa);
                if (!(fabs(lc - ela) > 1.0e-3 * width && fabs(lc - elb) > 1.0e-3 * width)) lc = 0.5 * (ela + elb);
                ec = exp(lc);
            }
        }
        if (eph != 9) {
            start_F(ec);
            return;
        }
        // the n_e root: the state of the last point evaluated
        passes += enev;
        ne = eb;
        xHI = Sb.x;
        xHeI = Sb.h1;
        xHeII = Sb.h2;
        req = kReqFinish;
    }
    // thermal_bracketed after net(t)
    __device__ void on_net(double f) {
        ++nev;
        tsr.feed(f, A->te_min, A->te_max);
        if (tsr.ph != 9) {
            start_net(tsr.t);
            return;
        }
        // the leaf's T_e; the written state (thermal_mod.f90:191-203)
        const BalArgs& b = A->b;
        te = tsr.tr;
        const double w = b.relax;
        xn = (1.0 - w) * x0 + w * xHI;
        h1n = (1.0 - w) * h10 + w * xHeI;
        h2n = (1.0 - w) * h20 + w * xHeII;
        const double h3n = fmax(0.0, 1.0 - h1n - h2n);
        nen_hhe = nH * ((1.0 - xn) + b.yHe * (h2n + 2.0 * h3n));
        nen = nen_hhe;
        req = kReqNone;
        if (b.metal_ne) {   // charge_neutrality_ne from the solved n_e
            in_neu = true;
            nit = 0;
            nen = fmax(ne, 1.0e-12 * nH);
            ask_sums(nen, xn);
        }
    }
    __device__ void on_neu(double em) {
        const double ne_old = nen;
        double v = nen_hhe + em;
        v = fmax(0.5 * (v + ne_old), 1.0e-12 * nH);
        nen = v;
        if (fabs(v - ne_old) <= 1.0e-10 * v || ++nit >= 200) {
            in_neu = false;
            req = kReqNone;
        } else {
            ask_sums(nen, xn);
        }
    }
};

__global__ void __launch_bounds__(kBThreads) k_thermal_flow(const ThArgs a, unsigned long long* next) {
    __shared__ double sh[6][kBThreads];
    const BalArgs& b = a.b;
    double mdx = 0.0, mdt = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
    unsigned long long solved = 0, tpass = 0, tsums = 0, nevals = 0;
    SerialCascade mc;
    mc.m = &b.m;
    LeafFlow L;
    L.A = &a;
    // the first leaf of each lane: its own position; then from the counter
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = b.nleaf;
    const long long first_claimed = (long long)gridDim.x * blockDim.x;
    for (;;) {
        // start leaves until one needs solving (empty leaves finish at once)
        while (!L.live && p < n) {
            const long long il = a.order ? (long long)a.order[n - 1 - p] : p;   // the most work first
            if (b.nH[il] <= 0.0) {
                b.ne[il] = 0.0;
                write_columns(b.col, il, b.nabs, b.fp32, b.nH[il], b.yHe, b.xHI[il], b.xHeI[il], b.xHeII[il],
                              b.colscale, b.rhokap ? b.rhokap[il] : 0.0);
                if (a.work) a.work[il] = 0u;
                p = first_claimed + (long long)atomicAdd(next, 1ull);
                continue;
            }
            L.start_leaf(p, il);
        }
        const unsigned live = __ballot_sync(kFull, L.live);
        if (!live) break;
        // the rate cache and the net heating are costly and asked for once per
        // trial T, so they are served when at least half the live lanes ask,
        // or when no live lane asks for a cascade sum
        const unsigned wp = __ballot_sync(kFull, L.live && L.req == kReqPrepare);
        const unsigned wf = __ballot_sync(kFull, L.live && L.req == kReqFinish);
        const unsigned ws = __ballot_sync(kFull, L.live && L.req == kReqSums);
        const int nl = __popc(live);
        const bool serve_p = wp && (2 * __popc(wp) >= nl || !ws);
        const bool serve_f = wf && (2 * __popc(wf) >= nl || !ws);
        if (serve_p) {
            if (L.live && L.req == kReqPrepare) {
                mc.prepare(L.il, L.q_T);
                L.on_prepare();
            }
        }
        if (__any_sync(kFull, L.live && L.req == kReqSums)) {
            if (L.live && L.req == kReqSums) {
                double nem, rin, rout;
                mc.sums(L.nH, L.q_ne, L.nH * L.q_x, L.nH * (1.0 - L.q_x), nem, rin, rout);
                L.on_sums(nem, rin, rout);
            }
        }
        if (serve_f) {
            if (L.live && L.req == kReqFinish) {
                const long long il = L.il;
                const long long nl = b.nleaf;
                const double heat = L.nH * (L.xHI * b.rates[3 * nl + il] +
                                            b.yHe * (L.xHeI * b.rates[4 * nl + il] + L.xHeII * b.rates[5 * nl + il]));
                double net = heat - cooling_total(a.td, b.rs, b.caseA, b.yHe, L.q_T, L.nH, L.ne, L.xHI, L.xHeI, L.xHeII);
                const MetalThermalTerms mt =
                    thermal_terms(a.td, mc, il, L.q_T, L.nH, L.ne, L.nH * L.xHI, L.nH * (1.0 - L.xHI));
                net = net - mt.cool;
                net = net - mt.cool_H;
                if (b.metal_ff) net = net - mt.freefree;
                if (b.metal_heat) net = net + mt.heat;
                L.on_net(net);
            }
        }
        // a lane whose leaf is solved writes it and takes the next one
        if (L.live && L.req == kReqNone) {
            const long long il = L.il;
            if (b.fp32) mc.opacity_fill<float>(il, L.nH, L.nen, L.xn, b.colscale);
            else mc.opacity_fill<double>(il, L.nH, L.nen, L.xn, b.colscale);
            ++solved;
            tpass += (unsigned long long)L.passes;
            tsums += (unsigned long long)L.nsum;
            nevals += (unsigned long long)L.nev;
            if (a.work) a.work[il] = (unsigned)min(L.nsum, 65535);
            b.xHI[il] = L.xn;
            b.xHeI[il] = L.h1n;
            b.xHeII[il] = L.h2n;
            b.ne[il] = L.nen;
            b.Te[il] = L.te;
            write_columns(b.col, il, b.nabs, b.fp32, L.nH, b.yHe, L.xn, L.h1n, L.h2n, b.colscale,
                          b.rhokap ? b.rhokap[il] : 0.0);
            const double dx = fabs(L.xn - L.x0);
            mdx = fmax(mdx, dx);
            mdt = fmax(mdt, fabs(L.te - L.T0) / L.T0);
            const double vol = leaf_vol(b, il);
            s1 = s1 + vol * dx;
            s2 = s2 + vol * (1.0 - L.xn);
            s3 = s3 + vol * L.nen * fabs(L.te - L.T0);
            s4 = s4 + vol * L.nen * L.te;
            L.live = false;
            p = first_claimed + (long long)atomicAdd(next, 1ull);
        }
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
        solved += __shfl_down_sync(kFull, solved, o);
        tpass += __shfl_down_sync(kFull, tpass, o);
        tsums += __shfl_down_sync(kFull, tsums, o);
        nevals += __shfl_down_sync(kFull, nevals, o);
    }
    if ((t & 31) == 0) {
        if (solved) atomicAdd(b.counters + 0, solved);
        if (tpass) atomicAdd(b.counters + 2, tpass);
        if (tsums) atomicAdd(b.counters + 3, tsums);
        if (nevals) atomicAdd(b.counters + 4, nevals);
    }
}

// gas_thermal_update with metals, one warp per leaf (WarpCascade): the
// same solve as k_thermal; lane 0 writes the leaf's state, the element lanes
// its opacity weights.  128-thread blocks, grid-stride over leaves by warps.
constexpr int kWThreads = 128;

__global__ void __launch_bounds__(kWThreads) k_thermal_warp(const ThArgs a) {
    __shared__ double sh[6][kWThreads / 32];
    const BalArgs& b = a.b;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double mdx = 0.0, mdt = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
    unsigned long long solved = 0, caps = 0, tpass = 0, tsums = 0, nevals = 0;
    WarpCascade mc;
    mc.init(b.m);
    const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long il = (long long)blockIdx.x * (blockDim.x >> 5) + wib; il < b.nleaf; il += nw) {
        const double nH = b.nH[il];
        const double x0 = b.xHI[il], h10 = b.xHeI[il], h20 = b.xHeII[il], T0 = b.Te[il];
        if (nH <= 0.0) {
            if (lane == 0) {
                b.ne[il] = 0.0;
                write_columns(b.col, il, b.nabs, b.fp32, nH, b.yHe, x0, h10, h20, b.colscale,
                              b.rhokap ? b.rhokap[il] : 0.0);
            }
            continue;
        }
        double xHI = x0, xHeI = h10, xHeII = h20, ne = 0.0;
        int passes = 0, nsum = 0, nev = 0, last = 0;
        double te;
        if (b.fast) {
            ne = b.ne[il];
            te = thermal_bracketed(a, il, nH, xHI, xHeI, xHeII, ne, &passes, mc, &nsum, &nev,
                                   a.Twarm ? a.Twarm[il] : T0);
        } else {
            double tlo = a.te_min, thi = a.te_max;
            nev = 3;
            const double net_lo = net_rate(a, il, tlo, nH, xHI, xHeI, xHeII, ne, &passes, mc, &nsum);
            const double net_hi = net_rate(a, il, thi, nH, xHI, xHeI, xHeII, ne, &passes, mc, &nsum);
            if (net_lo <= 0.0) {
                te = tlo;
            } else if (net_hi >= 0.0) {
                te = thi;
            } else {
                for (int it = 1; it <= 60; ++it) {
                    const double tmid = sqrt(tlo * thi);
                    const double nm = net_rate(a, il, tmid, nH, xHI, xHeI, xHeII, ne, &passes, mc, &nsum);
                    ++nev;
                    if (nm > 0.0) tlo = tmid; else thi = tmid;
                    if (thi / tlo - 1.0 < 1.0e-5) break;
                }
                te = sqrt(tlo * thi);
            }
            net_rate(a, il, te, nH, xHI, xHeI, xHeII, ne, &last, mc, &nsum);
            if (last > 200) ++caps;
        }
        ++solved;
        tpass += (unsigned long long)(passes + last);
        tsums += (unsigned long long)nsum;
        nevals += (unsigned long long)nev;
        const double w = b.relax;
        const double xn = (1.0 - w) * x0 + w * xHI;
        const double h1n = (1.0 - w) * h10 + w * xHeI;
        const double h2n = (1.0 - w) * h20 + w * xHeII;
        const double h3n = fmax(0.0, 1.0 - h1n - h2n);
        double nen = nH * ((1.0 - xn) + b.yHe * (h2n + 2.0 * h3n));
        // written state at te (thermal_mod.f90:191-203); the cascade is at te
        // from the final net_rate
        if (b.metal_ne) nen = charge_neutrality_ne(mc, nH, nen, xn, ne);
        if (b.fp32) mc.opacity_fill<float>(il, nH, nen, xn, b.colscale);
        else mc.opacity_fill<double>(il, nH, nen, xn, b.colscale);
        if (lane == 0) {
            b.xHI[il] = xn;
            b.xHeI[il] = h1n;
            b.xHeII[il] = h2n;
            b.ne[il] = nen;
            b.Te[il] = te;
            write_columns(b.col, il, b.nabs, b.fp32, nH, b.yHe, xn, h1n, h2n, b.colscale,
                          b.rhokap ? b.rhokap[il] : 0.0);
        }
        const double dx = fabs(xn - x0);
        mdx = fmax(mdx, dx);
        mdt = fmax(mdt, fabs(te - T0) / T0);
        const double vol = leaf_vol(b, il);
        s1 = s1 + vol * dx;
        s2 = s2 + vol * (1.0 - xn);
        s3 = s3 + vol * nen * fabs(te - T0);
        s4 = s4 + vol * nen * te;
    }
    // every lane of a warp holds the same sums; lane 0 reports them
    if (lane == 0) {
        sh[0][wib] = mdx; sh[1][wib] = mdt; sh[2][wib] = s1; sh[3][wib] = s2; sh[4][wib] = s3; sh[5][wib] = s4;
        if (solved) atomicAdd(b.counters + 0, solved);
        if (caps) atomicAdd(b.counters + 1, caps);
        if (tpass) atomicAdd(b.counters + 2, tpass);
        if (tsums) atomicAdd(b.counters + 3, tsums);
        if (nevals) atomicAdd(b.counters + 4, nevals);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r[6] = {sh[0][0], sh[1][0], sh[2][0], sh[3][0], sh[4][0], sh[5][0]};
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            r[0] = fmax(r[0], sh[0][w]);
            r[1] = fmax(r[1], sh[1][w]);
            for (int k = 2; k < 6; ++k) r[k] = r[k] + sh[k][w];
        }
        for (int k = 0; k < 6; ++k) b.partial[6 * blockIdx.x + k] = r[k];
    }
}

// Stage fractions of the written state (species_write, species_mod.f90:873-904):
// leaf-major, registry order; an empty leaf is all neutral.
__global__ void k_metal_fractions(const MetalDev m, const double* __restrict__ nH, const double* __restrict__ xHI,
                                  const double* __restrict__ ne, const double* __restrict__ Te, long long nleaf,
                                  double* out) {
    for (long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x; il < nleaf;
         il += (long long)gridDim.x * blockDim.x) {
        double* o = out + il * m.nst;
        if (nH[il] <= 0.0) {
            for (int ie = 0; ie < m.nel; ++ie) {
                const MetalEl e = m.el[ie];
                for (int i = 0; i < e.nstage; ++i) o[e.st0 + i] = i == 0 ? 1.0 : 0.0;
            }
            continue;
        }
        MetalCache mc;
        metal_prepare(m, il, Te[il], mc);
        const double nHI = nH[il] * xHI[il], nHII = nH[il] * (1.0 - xHI[il]);
        double r[kMaxSt];
        for (int ie = 0; ie < m.nel; ++ie) {
            const MetalEl e = m.el[ie];
            double fr = metal_chain(mc, e.tr0, e.nstage, ne[il], nHI, nHII, r);
            o[e.st0] = fr;
            for (int i = 2; i <= e.nstage; ++i) {
                fr = fr * r[i - 2];
                o[e.st0 + i - 1] = fr;
            }
        }
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
        c->nH, c->xHI, c->xHeI, c->xHeII, c->ne, c->Te, c->col, c->grid.nleaf, c->nabs, c->fp32 ? 1 : 0,
        c->par.He_abund, c->par.distance2cm * 1.0e-18, c->metal, c->rhokap);
    return cudaGetLastError();
}

cudaError_t launch_metal_fractions(mochii_ctx* c, double* out) {
    k_metal_fractions<<<nblocks(c->grid.nleaf, 128, 148 * 16), 128, 0, c->stream>>>(c->metal, c->nH, c->xHI, c->ne,
                                                                                   c->Te, c->grid.nleaf, out);
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
    a.lg = c->oct.ncells > 0 ? c->oct.lgeo : nullptr;
    a.rhokap = c->rhokap;
    a.rs.hui_gnedin = c->par.recomb_hui_gnedin;
    a.rs.dere_hybrid = c->par.ci_dere_hybrid;
    a.caseA = c->par.caseA;
    a.nabs = c->nabs;
    a.fp32 = c->fp32 ? 1 : 0;
    a.k = coef_at(a.rs, a.caseA, a.T);   // fixed T: evaluated once on the host
    a.m = c->metal;
    a.metal_ne = c->par.metal_ne;
    a.two_way = c->par.charge_exchange_two_way;
    a.metal_heat = c->par.metal_heat;
    a.metal_ff = c->par.metal_freefree;
    a.fast = c->par.solver_bracketed;
    a.nemax = 1.0 + 2.0 * c->par.He_abund;
    for (const MetalEl& e : c->species.el) a.nemax += e.abund * (double)(e.nstage - 1);
    return a;
}

cudaError_t nl_log_tables(const double* lamref, const double* Ssup, int ntab, double** out, cudaStream_t s) {
    cudaError_t e = cudaMalloc(out, (size_t)ntab * kNlNT * kNlNNE * 8);
    if (e != cudaSuccess) return e;
    k_nl_log<<<nblocks((long long)ntab * kNlNT * kNlNNE, 256, 148 * 16), 256, 0, s>>>(lamref, Ssup, ntab, *out);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return cudaStreamSynchronize(s);
}

cudaError_t metal_ttable_build(mochii_ctx* c) {
    MetalDev& m = c->metal;
    const int nt = 4096;
    const double u0 = log(c->par.te_min), u1 = log(c->par.te_max);
    m.tnt = 0;
    m.tdu = (u1 - u0) / (double)(nt - 6);
    m.tu0 = u0 - 3.0 * m.tdu;
    double* t = nullptr;
    // one allocation: the rate coefficients (ntr x 4 x nt), then the cooling fits (nst x nt)
    cudaError_t e = cudaMalloc(&t, ((size_t)m.ntr * 4 + m.nst) * nt * 8);
    if (e != cudaSuccess) return e;
    c->ttab = t;
    MetalDev mb = m;
    mb.tnt = nt;
    double* ct = t + (size_t)m.ntr * 4 * nt;
    k_metal_ttable<<<nblocks((long long)m.ntr * 4 * nt, 256, 148 * 16), 256, 0, c->stream>>>(mb, t);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (m.nst > 0) k_metal_ctable<<<nblocks((long long)m.nst * nt, 256, 148 * 16), 256, 0, c->stream>>>(mb, ct);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return e;
    m.ttab = t;
    m.ctab = ct;
    m.tnt = nt;
    return cudaSuccess;
}

cudaError_t launch_balance(mochii_ctx* c) {
    const BalArgs a = bal_args(c);
    k_balance<<<c->bw.blocks, kBThreads, 0, c->stream>>>(a);
    return cudaGetLastError();
}

// The work-order buffers of the lockstep solve (sorted leaves, chunk counter).
cudaError_t thermal_work_alloc(mochii_ctx* c) {
    BalanceWork& w = c->bw;
    const int n = (int)c->grid.nleaf;
    cudaError_t e;
    if ((e = cudaMalloc(&w.work, (size_t)n * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.work_sorted, (size_t)n * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.iota, (size_t)n * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.order, (size_t)n * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&w.next, sizeof(unsigned long long))) != cudaSuccess) return e;
    cub::DeviceRadixSort::SortPairs(nullptr, w.sort_bytes, w.work, w.work_sorted, w.iota, w.order, n, 0, 16);
    if ((e = cudaMalloc(&w.sort_tmp, w.sort_bytes)) != cudaSuccess) return e;
    k_iota<<<nblocks(n, 256, 148 * 16), 256, 0, c->stream>>>(w.iota, n);
    w.have_work = false;
    return cudaGetLastError();
}

// Launch shape of k_thermal_lane: the cache slots per lane decide how many
// lanes fit in shared memory; one block per SM (at most kBThreads threads,
// at least one warp), never more blocks than the balance's partial slots.
cudaError_t thermal_lane_setup(mochii_ctx* c) {
    BalanceWork& w = c->bw;
    int nslot = 0;
    for (const MetalTr& t : c->species.tr) nslot += lane_slots(lane_kind(t));
    int smem_max = 0, sms = 148;
    cudaError_t e = cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    if (e != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device)) != cudaSuccess) return e;
    const size_t fixed = lane_cache_offset() + 6 * (kBThreads / 32) * 8 + 1024;   // layout, reduction, reserve
    const size_t per_lane = (size_t)std::max(nslot, 1) * 8;
    int threads = (int)(((size_t)smem_max - fixed) / per_lane) / 32 * 32;
    threads = std::max(32, std::min(kBThreads, threads));
    if (c->tune.lane_threads > 0) threads = std::max(32, std::min(threads, c->tune.lane_threads / 32 * 32));   // the cell tile
    w.lane_threads = threads;
    w.lane_smem = lane_cache_offset() + per_lane * threads;
    w.lane_blocks = std::max(1, std::min(sms, c->bw.blocks));
    e = cudaFuncSetAttribute(k_thermal_lane, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)w.lane_smem);
    if (e != cudaSuccess) {
        w.lane_threads = 0;
        return e;
    }
    return cudaSuccess;
}

// ---- batched nebulae --------------------------------------------------------
struct ThermalBatch {
    std::vector<ThArgs> h_args;             // host copy of d_args
    ThArgs* d_args = nullptr;
    long long* d_off = nullptr;
    unsigned long long* d_next = nullptr;   // lockstep: one chunk counter; lane: one leaf counter per nebula
    int n = 0, blocks = 0;
    bool lane = false;                      // the per-lane solve (cell_layout 'lane')
    int threads = kBThreads;
    size_t smem = 0;
};

void* thermal_batch_create(mochii_ctx* const* cs, int n, cudaError_t* err) {
    *err = cudaSuccess;
    auto* tb = new ThermalBatch();
    tb->n = n;
    std::vector<ThArgs> args(n);
    std::vector<long long> off(n + 1, 0);
    for (int k = 0; k < n; ++k) {
        mochii_ctx* c = cs[k];
        if (!c->bw.work && (*err = thermal_work_alloc(c)) != cudaSuccess) break;
        // a zero work array sorts to a valid order: the graph always sorts
        if ((*err = cudaMemsetAsync(c->bw.work, 0, (size_t)c->grid.nleaf * 4, c->stream)) != cudaSuccess) break;
        c->bw.have_work = true;
        ThArgs& a = args[k];
        a.b = bal_args(c);
        a.td = c->th;
        a.te_min = c->par.te_min;
        a.te_max = c->par.te_max;
        a.Twarm = nullptr;
        a.tfac0 = 1.05;
        a.gate = 0.0;
        a.order = c->bw.order;
        a.work = c->bw.work;
        a.next = nullptr;
        off[k + 1] = off[k] + (c->grid.nleaf + 31) / 32;
        if ((*err = cudaStreamSynchronize(c->stream)) != cudaSuccess) break;
    }
    if (*err == cudaSuccess) *err = cudaMalloc(&tb->d_args, sizeof(ThArgs) * n);
    if (*err == cudaSuccess) *err = cudaMalloc(&tb->d_off, sizeof(long long) * (n + 1));
    tb->lane = cs[0]->par.solver_warp == 3;
    if (*err == cudaSuccess) *err = cudaMalloc(&tb->d_next, sizeof(unsigned long long) * (tb->lane ? n : 1));
    if (*err == cudaSuccess) *err = cudaMemcpy(tb->d_args, args.data(), sizeof(ThArgs) * n, cudaMemcpyHostToDevice);
    tb->h_args = args;
    if (*err == cudaSuccess) *err = cudaMemcpy(tb->d_off, off.data(), sizeof(long long) * (n + 1), cudaMemcpyHostToDevice);
    if (*err == cudaSuccess && tb->lane) {   // shared cache sized to the largest nebula's slots
        int nslot = 1, smem_max = 0, sms = 148;
        for (int k = 0; k < n; ++k) {
            int q = 0;
            for (const MetalTr& t : cs[k]->species.tr) q += lane_slots(lane_kind(t));
            nslot = std::max(nslot, q);
        }
        cudaFuncAttributes fa;
        *err = cudaFuncGetAttributes(&fa, k_thermal_lane_batch);
        if (*err == cudaSuccess) *err = cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                                               cs[0]->device);
        if (*err == cudaSuccess) *err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cs[0]->device);
        if (*err == cudaSuccess) {
            const size_t avail = (size_t)smem_max - fa.sharedSizeBytes - 1024;
            int threads = (int)(avail / ((size_t)nslot * 8)) / 32 * 32;
            tb->threads = std::max(32, std::min(kBThreads, threads));
            tb->smem = (size_t)nslot * 8 * tb->threads;
            tb->blocks = sms;
            *err = cudaFuncSetAttribute(k_thermal_lane_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)tb->smem);
        }
    } else if (*err == cudaSuccess) {
        int per = 1, sms = 148;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_thermal_batch, kBThreads, 0);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cs[0]->device);
        tb->blocks = std::max(1, per) * sms;
    }
    if (*err != cudaSuccess) {
        thermal_batch_destroy(tb);
        return nullptr;
    }
    return tb;
}

void thermal_batch_destroy(void* p) {
    auto* tb = static_cast<ThermalBatch*>(p);
    if (!tb) return;
    for (void* q : {(void*)tb->d_args, (void*)tb->d_off, (void*)tb->d_next})
        if (q) cudaFree(q);
    delete tb;
}

// The learned warm start in the batched thermal update: nebula k's solve
// starts from cs[k]->twarm with the first step fac[k] and the residual gate.
cudaError_t thermal_batch_set_warm(void* p, mochii_ctx* const* cs, const double* fac, double gate) {
    auto* tb = static_cast<ThermalBatch*>(p);
    for (int k = 0; k < tb->n; ++k) {
        tb->h_args[k].Twarm = cs[k]->twarm;
        tb->h_args[k].tfac0 = fac[k];
        tb->h_args[k].gate = gate;
    }
    return cudaMemcpy(tb->d_args, tb->h_args.data(), sizeof(ThArgs) * tb->n, cudaMemcpyHostToDevice);
}

// One batched thermal update on stream s: each nebula's leaves sorted by
// their last work and its sums cleared, then one persistent launch.
cudaError_t thermal_batch_enqueue(void* p, mochii_ctx* const* cs, cudaStream_t s) {
    auto* tb = static_cast<ThermalBatch*>(p);
    cudaError_t e;
    for (int k = 0; k < tb->n; ++k) {
        mochii_ctx* c = cs[k];
        BalanceWork& w = c->bw;
        const int n = (int)c->grid.nleaf;
        if ((e = cudaMemsetAsync(w.counters, 0, 8 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(w.partial, 0, 6 * (size_t)w.blocks * 8, s)) != cudaSuccess) return e;
        e = cub::DeviceRadixSort::SortPairs(w.sort_tmp, w.sort_bytes, w.work, w.work_sorted, w.iota, w.order, n, 0, 16, s);
        if (e != cudaSuccess) return e;
    }
    if (tb->lane) {
        if ((e = cudaMemsetAsync(tb->d_next, 0, sizeof(unsigned long long) * tb->n, s)) != cudaSuccess) return e;
        k_thermal_lane_batch<<<tb->blocks, tb->threads, tb->smem, s>>>(tb->d_args, tb->n, tb->d_next);
        return cudaGetLastError();
    }
    if ((e = cudaMemsetAsync(tb->d_next, 0, sizeof(unsigned long long), s)) != cudaSuccess) return e;
    k_thermal_batch<<<tb->blocks, kBThreads, 0, s>>>(tb->d_args, tb->n, tb->d_off, tb->d_next);
    return cudaGetLastError();
}

cudaError_t launch_thermal(mochii_ctx* c) {
    ThArgs a;
    a.b = bal_args(c);
    a.td = c->th;
    a.te_min = c->par.te_min;
    a.te_max = c->par.te_max;
    a.Twarm = c->twarm_set ? c->twarm : nullptr;
    a.tfac0 = c->twarm_set ? c->twarm_fac : 1.05;
    a.gate = c->twarm_set ? c->twarm_gate : 0.0;
    a.order = nullptr;
    a.work = nullptr;
    a.next = nullptr;
    if (c->metal.ntr > 0 && c->par.solver_warp == 1) {
        k_thermal_warp<<<c->bw.blocks, kWThreads, 0, c->stream>>>(a);
    } else if (c->metal.ntr > 0 && c->par.solver_bracketed) {
        BalanceWork& w = c->bw;
        const int n = (int)c->grid.nleaf;
        cudaError_t e;
        if (!w.work && (e = thermal_work_alloc(c)) != cudaSuccess) return e;
        if (w.have_work) {
            e = cub::DeviceRadixSort::SortPairs(w.sort_tmp, w.sort_bytes, w.work, w.work_sorted, w.iota, w.order, n, 0,
                                                16, c->stream);
            if (e != cudaSuccess) return e;
            a.order = w.order;
        }
        a.work = w.work;
        if (c->par.solver_warp == 2) {
            if ((e = cudaMemsetAsync(w.next, 0, sizeof(unsigned long long), c->stream)) != cudaSuccess) return e;
            k_thermal_flow<<<c->bw.blocks, kBThreads, 0, c->stream>>>(a, w.next);
        } else if (c->par.solver_warp == 3) {
            if (w.lane_threads == 0 && (e = thermal_lane_setup(c)) != cudaSuccess) return e;
            if ((e = cudaMemsetAsync(w.next, 0, sizeof(unsigned long long), c->stream)) != cudaSuccess) return e;
            if ((e = cudaMemsetAsync(c->bw.partial, 0, 6 * (size_t)c->bw.blocks * 8, c->stream)) != cudaSuccess) return e;
            a.next = w.next;
            k_thermal_lane<<<w.lane_blocks, w.lane_threads, w.lane_smem, c->stream>>>(a);
        } else {
            if (w.ls_blocks == 0) {   // persistent: the resident blocks of the device
                int per = 1, sms = 148;
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_thermal_ls, kBThreads, 0);
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
                w.ls_blocks = std::max(1, std::min(c->bw.blocks, std::max(per, 1) * sms));
            }
            if ((e = cudaMemsetAsync(w.next, 0, sizeof(unsigned long long), c->stream)) != cudaSuccess) return e;
            if ((e = cudaMemsetAsync(c->bw.partial, 0, 6 * (size_t)c->bw.blocks * 8, c->stream)) != cudaSuccess) return e;
            a.next = w.next;
            k_thermal_ls<<<w.ls_blocks, kBThreads, 0, c->stream>>>(a);
        }
        w.have_work = true;
    } else {
        k_thermal<<<c->bw.blocks, kBThreads, 0, c->stream>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace mochii
