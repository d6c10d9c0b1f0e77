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
#include "transport.h"

namespace mochii {

namespace {

constexpr int kBThreads = 256;

struct BalArgs {
    const double* nH;
    double* xHI;
    double* xHeI;
    double* xHeII;
    double* ne;
    const double* Te;
    const double* rates;   // gamma_HI, gamma_HeI, gamma_HeII, heat_* (6 x nleaf)
    void* col;
    double* partial;
    unsigned long long* counters;
    long long nleaf;
    double T, yHe, relax, colscale, vol;
    RateSel rs;
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

// solve_ion_cell on the H/He path (no metal electrons, no charge exchange):
// returns the number of fixed-point passes used.
__device__ int solve_cell(const RateSel& rs, double yHe, double gH, double gHe1, double gHe2, double nH, double T,
                          int caseA, double& xHI, double& xHeI, double& xHeII, double& ne) {
    const double aH = caseA ? alphaA_HII(rs, T) : alphaB_HII(rs, T);
    const double aHe2 = caseA ? alphaA_HeII(rs, T) : alphaB_HeII(rs, T);
    const double aHe3 = caseA ? alphaA_HeIII(rs, T) : alphaB_HeIII(rs, T);
    const double cH = ci_HI(rs, T), cHe1 = ci_HeI(rs, T), cHe2 = ci_HeII(rs, T);
    double xHeIII = fmax(0.0, 1.0 - xHeI - xHeII);
    ne = nH * ((1.0 - xHI) + yHe * (xHeII + 2.0 * xHeIII));
    ne = fmax(ne, 1.0e-12 * nH);
    int it = 1;
    for (; it <= 200; ++it) {
        const double ne_old = ne;
        const double denH = gH + (cH + aH) * ne + 0.0 + 0.0;
        xHI = denH > 0.0 ? (aH * ne + 0.0) / denH : 1.0;
        const double r1 = fmin((gHe1 + cHe1 * ne) / (aHe2 * ne), 1.0e150);
        const double r2 = fmin((gHe2 + cHe2 * ne) / (aHe3 * ne), 1.0e150);
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
        const int it = solve_cell(a.rs, a.yHe, a.rates[il], a.rates[a.nleaf + il], a.rates[2 * a.nleaf + il], nH,
                                  a.T, a.caseA, xHI, xHeI, xHeII, ne);
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

cudaError_t launch_balance(mochii_ctx* c) {
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
    k_balance<<<c->bw.blocks, kBThreads, 0, c->stream>>>(a);
    return cudaGetLastError();
}

}  // namespace mochii
