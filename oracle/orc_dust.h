// Oracle (test infrastructure only): grain optics of the ionizing band and
// the random stream of the scattered flights.
//
// DustTable restates gas_opacity_mod.f90: the extinction-table read
// (ion_dust_read :69-121: numeric rows "lambda albedo <cos> C_ext/H ...",
// sorted ascending in lambda by a stable insertion sort :258-275), the
// interpolators interp_log / interp_lin (:277-315) and the exact-energy
// evaluators ion_dust_sabs_at / ssca_at / g_at (:231-256).
//
// Philox restates the counter-based generator Philox4x32-10 of Salmon,
// Moraes, Dror & Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC11).
// The reference draws its scattering numbers from a per-rank MT19937 stream
// (random.f90 rand_number); the device cannot reproduce a sequential
// stream per packet, so both the oracle and the device draw from Philox
// keyed by (par%iseed, packet stream) with the packet index in the counter:
// the n-th draw of a packet is the same number on both.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

namespace orc {

struct DustTable {
    std::vector<double> lam, alb, gcos, cext;   // ascending lambda [um]
    double cref = 0.0;                          // C_ext at lambda_ref
    bool read(const std::string& path, double lambda_ref, std::string* err);
    double sabs_at(double E) const;             // (1 - albedo) C_ext / C_ref at lambda = 1.23984/E
    double ssca_at(double E) const;             // albedo C_ext / C_ref
    double g_at(double E) const;                // <cos>
};

// dust_temp_mod.f90:38-170: the equilibrium mixture dust temperature's
// emission function femit(T) = 4 pi Int s_abs B_nu dnu (trapezoid on the
// table's frequency grid) on 61 log T nodes, s_abs at 240 log IR wavelengths
// (1 - 1000 um), and the per-leaf root of Heat_dust = kd femit(T).
struct DustTemp {
    static constexpr int NT = 61, NIR = 240;
    double tgrid[NT], femit[NT], lam_ir[NIR], sabs_ir[NIR];
    void setup(const DustTable& d);
    double femit_of(double T) const;
    double solve(double kd, double heat) const;   // 0 where kd or heat is not positive
};
double planck_nu(double nu, double T);

double interp_log(const std::vector<double>& x, const std::vector<double>& y, double x0);
double interp_lin(const std::vector<double>& x, const std::vector<double>& y, double x0);
// One Fortran list-directed real (1.5, 1.5E+3, 1.5D3, 1.5-3 = 1.5E-3).
bool fortran_real(const std::string& tok, double* v);

// The n-th uniform in (0, 1) of one packet's stream: two 32-bit words of
// the Philox4x32-10 block n/2 (counter = (n/2, 0, packet lo, packet hi),
// key = (seed lo, seed hi ^ stream)), 53 bits.
double philox_uniform(uint64_t seed, uint32_t stream, uint64_t packet, uint32_t n);
// One Philox4x32-10 block: ctr[4], key[2] -> out[4].
void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

struct PacketRng {
    uint64_t seed = 0, packet = 0;
    uint32_t stream = 0, n = 0;
    double next() { return philox_uniform(seed, stream, packet, n++); }
};

}  // namespace orc
