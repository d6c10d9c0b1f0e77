// Grain optics of the ionizing band (gas_opacity_mod.f90) and the random
// stream of the scattered flights.
//
// Host: the extinction table par%ion_dust_kext (ion_dust_read, :69-121):
// the rows of four leading reals "lambda [um]  albedo  <cos>  C_ext/H" with
// lambda > 0, sorted ascending in lambda (stable, as sort4 :258-275), and
// C_ext at par%lambda_ref.  Device: the exact-energy evaluators
// ion_dust_sabs_at / ssca_at / g_at (:231-256) over one copy of the table
// (5 x n doubles), the interpolation bracket found by a binary search that
// returns the bracket the reference's linear scan returns.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace mochii {

struct DustHost {
    std::vector<double> lam, alb, gcos, cext;
    double cref = 0.0;
};

// Read and sort the table; false with *err on failure.
bool dust_table_read(const std::string& path, double lambda_ref, DustHost& d, std::string* err);

struct DustDev {
    int n = 0;                      // 0: no grain optics
    const double* lam = nullptr;    // ascending [um]
    const double* alb = nullptr;
    const double* gcos = nullptr;
    const double* cext = nullptr;
    double cref = 0.0;
};

// The equilibrium dust temperature's tables (dust_temp_mod.f90:38-115):
// femit(T) on 61 log nodes of T (10^0.5 .. 10^3.5 K) and s_abs at 240 log
// wavelengths from 1 to 1000 um.
constexpr int kDustTN = 61, kDustIrN = 240;
struct DustTempHost {
    double tgrid[kDustTN] = {}, femit[kDustTN] = {};
    double lam_ir[kDustIrN] = {}, sabs_ir[kDustIrN] = {};
};
void dust_temp_tables(const DustHost& d, DustTempHost& t);

}  // namespace mochii
