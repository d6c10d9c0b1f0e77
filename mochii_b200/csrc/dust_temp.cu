// Equilibrium dust temperature and the grains' infrared spectrum from the
// grain heating of the last transport pass (dust_temp_mod.f90).
//
// Host: the emission function femit(T) = 4 pi Int s_abs(nu) B_nu(T) dnu over
// the extinction table the transport uses (trapezoid on the table's own
// frequency grid, s_abs = (1 - albedo) C_ext / C_ext(lambda_ref)) on 61 log
// nodes of T from 10^0.5 to 10^3.5 K, and s_abs on 240 log wavelengths from
// 1 to 1000 um (dust_temp_setup, :38-115).  Device: per leaf the root of
// Heat_dust = (rhokap / d_cm) femit(T) by bisection in ln T
// (dust_temp_compute, :137-170), and the grid-integrated modified blackbody
// L_nu = sum_leaf 4 pi (rhokap / d_cm) s_abs(nu) B_nu(T_d) V with the
// absorbed power sum Heat_dust V (dust_ir_write, :173-214).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "ctx.h"
#include "dust.h"
#include "transport.h"

namespace mochii {

namespace {

constexpr double kHplanck = 6.62607015e-27, kKb = 1.380649e-16, kClight = 2.99792458e10;
constexpr double kFourPi = 12.566370614359172953850573533118;

__host__ __device__ double planck_nu(double nu, double T) {
    const double x = kHplanck * nu / (kKb * T);
    return x < 700.0 ? 2.0 * kHplanck * nu * nu * nu / (kClight * kClight) / (exp(x) - 1.0) : 0.0;
}

double lin_interp(const std::vector<double>& x, const std::vector<double>& y, double x0) {
    const size_t n = x.size();
    if (x0 <= x[0]) return y[0];
    if (x0 >= x[n - 1]) return y[n - 1];
    size_t i = 0;
    while (i < n - 2 && !(x0 < x[i + 1])) ++i;
    const double w = (x0 - x[i]) / (x[i + 1] - x[i]);
    return y[i] * (1.0 - w) + y[i + 1] * w;
}

double log_interp(const std::vector<double>& x, const std::vector<double>& y, double x0) {
    const size_t n = x.size();
    if (x0 <= x[0]) return y[0];
    if (x0 >= x[n - 1]) return y[n - 1];
    size_t i = 0;
    while (i < n - 2 && !(x0 < x[i + 1])) ++i;
    const double w = std::log(x0 / x[i]) / std::log(x[i + 1] / x[i]);
    return std::exp(std::log(std::max(y[i], 2.2250738585072014e-308)) * (1.0 - w) +
                    std::log(std::max(y[i + 1], 2.2250738585072014e-308)) * w);
}

// The tables: T nodes, femit, their log10 / ln (what the device reads), the
// IR wavelengths and s_abs there.
struct TempTab {
    double lg[kDustTN], lnf[kDustTN];
};

__device__ double femit_ln(const TempTab& t, double T) {
    const double lt = fmin(fmax(log10(T), t.lg[0]), t.lg[kDustTN - 1]);
    const int i = min((int)((lt - t.lg[0]) / (3.0 / (double)(kDustTN - 1))), kDustTN - 2);
    const double w = (lt - t.lg[i]) / (t.lg[i + 1] - t.lg[i]);
    return exp(t.lnf[i] * (1.0 - w) + t.lnf[i + 1] * w);
}

__global__ void k_dust_temp(long long n, const double* __restrict__ rhokap, const double* __restrict__ heat,
                            double d2cm, const TempTab t, double tlo0, double thi0, double* __restrict__ td) {
    for (long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x; il < n;
         il += (long long)gridDim.x * blockDim.x) {
        const double kd = rhokap[il] / d2cm;   // n_d C_ext(lambda_ref) [cm^-1]
        const double h = heat[il];
        double T = 0.0;
        if (kd > 0.0 && h > 0.0) {
            const double target = h / kd;
            double tlo = tlo0, thi = thi0;
            if (femit_ln(t, thi) <= target) {
                T = thi;
            } else {
                for (int it = 0; it < 60; ++it) {
                    const double tm = sqrt(tlo * thi);
                    if (femit_ln(t, tm) < target) tlo = tm;
                    else thi = tm;
                    if (thi / tlo - 1.0 < 1.0e-5) break;
                }
                T = sqrt(tlo * thi);
            }
        }
        td[il] = T;
    }
}

// L_nu at wavelength blockIdx.y (and, in row kDustIrN, the absorbed power):
// each thread sums its leaves, the block reduces, one atomic per block.
__global__ void k_dust_ir(long long n, const double* __restrict__ rhokap, const double* __restrict__ heat,
                          const double* __restrict__ td, const double4* __restrict__ lg, double vol0, double d2cm,
                          const double* __restrict__ lam_ir, const double* __restrict__ sabs_ir,
                          double* __restrict__ out) {
    __shared__ double red[256 / 32];
    const int k = blockIdx.y;
    double nu = 0.0, s = 0.0;
    if (k < kDustIrN) {
        nu = kClight / (lam_ir[k] * 1.0e-4);
        s = sabs_ir[k];
    }
    double acc = 0.0;
    for (long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x; il < n;
         il += (long long)gridDim.x * blockDim.x) {
        const double T = td[il];
        if (T <= 0.0) continue;
        double vol = vol0;
        if (lg) {
            const double w = 2.0 * lg[il].w * d2cm;
            vol = w * w * w;
        }
        if (k < kDustIrN) acc += kFourPi * (rhokap[il] / d2cm) * s * planck_nu(nu, T) * vol;
        else acc += heat[il] * vol;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += red[w];
        atomicAdd(out + k, b);
    }
}

}  // namespace

void dust_temp_tables(const DustHost& d, DustTempHost& t) {
    const std::vector<double>& lam = d.lam;
    const size_t n = lam.size();
    for (int i = 0; i < kDustTN; ++i) {
        t.tgrid[i] = std::pow(10.0, 0.5 + 3.0 * (double)i / (double)(kDustTN - 1));
        const double T = t.tgrid[i];
        double f = 0.0;
        for (size_t k = 0; k + 1 < n; ++k) {
            const double nu1 = kClight / (lam[k + 1] * 1.0e-4), nu2 = kClight / (lam[k] * 1.0e-4);
            const double snu = 0.5 * ((1.0 - d.alb[k]) * d.cext[k] + (1.0 - d.alb[k + 1]) * d.cext[k + 1]) / d.cref;
            const double bnu = 0.5 * (planck_nu(nu1, T) + planck_nu(nu2, T));
            f = f + kFourPi * snu * bnu * (nu2 - nu1);
        }
        t.femit[i] = f;
    }
    for (int k = 0; k < kDustIrN; ++k) {
        t.lam_ir[k] = std::exp(std::log(1.0) + (std::log(1000.0) - std::log(1.0)) * (double)k / (double)(kDustIrN - 1));
        t.sabs_ir[k] = (1.0 - lin_interp(lam, d.alb, t.lam_ir[k])) * log_interp(lam, d.cext, t.lam_ir[k]) / d.cref;
    }
}

// T_dust of every leaf into c->tdust (allocated on first use).
cudaError_t dust_temp_launch(mochii_ctx* c) {
    const long long n = c->grid.nleaf;
    cudaError_t e;
    if (!c->tdust) {
        DustTempHost h;
        dust_temp_tables(c->dust_host, h);
        if ((e = cudaMalloc(&c->tdust, (size_t)n * 8)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&c->tdust_tab, (size_t)(2 * kDustIrN + 2 * kDustTN) * 8)) != cudaSuccess) return e;
        std::vector<double> blob(2 * kDustIrN + 2 * kDustTN);
        std::copy(h.lam_ir, h.lam_ir + kDustIrN, blob.begin());
        std::copy(h.sabs_ir, h.sabs_ir + kDustIrN, blob.begin() + kDustIrN);
        std::copy(h.tgrid, h.tgrid + kDustTN, blob.begin() + 2 * kDustIrN);
        std::copy(h.femit, h.femit + kDustTN, blob.begin() + 2 * kDustIrN + kDustTN);
        if ((e = cudaMemcpy(c->tdust_tab, blob.data(), blob.size() * 8, cudaMemcpyHostToDevice)) != cudaSuccess)
            return e;
        c->tdust_host = h;
    }
    TempTab t;
    for (int i = 0; i < kDustTN; ++i) {
        t.lg[i] = std::log10(c->tdust_host.tgrid[i]);
        t.lnf[i] = std::log(c->tdust_host.femit[i]);
    }
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_dust_temp<<<std::max(blocks, 1), 256, 0, c->stream>>>(n, c->rhokap, c->rates + 6 * (size_t)n,
                                                           c->par.distance2cm, t, c->tdust_host.tgrid[0],
                                                           c->tdust_host.tgrid[kDustTN - 1], c->tdust);
    return cudaGetLastError();
}

// The IR spectrum of the current T_dust: out[k] = L_nu at lam_ir[k] (240),
// out[240] = the absorbed power sum Heat_dust V.
cudaError_t dust_ir_launch(mochii_ctx* c, double* out_dev) {
    const long long n = c->grid.nleaf;
    cudaError_t e = cudaMemsetAsync(out_dev, 0, (kDustIrN + 1) * 8, c->stream);
    if (e != cudaSuccess) return e;
    const double w = c->grid.dcell * c->par.distance2cm;
    dim3 grid((unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148)), kDustIrN + 1);
    k_dust_ir<<<grid, 256, 0, c->stream>>>(n, c->rhokap, c->rates + 6 * (size_t)n, c->tdust,
                                           c->oct.ncells > 0 ? c->oct.lgeo : nullptr, w * w * w,
                                           c->par.distance2cm, c->tdust_tab, c->tdust_tab + kDustIrN, out_dev);
    return cudaGetLastError();
}

}  // namespace mochii
