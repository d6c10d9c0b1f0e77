// Trace-metal registry (species_mod.f90): host parser and the device layout.
//
// Transitions are kept in two orders.  Element order (j) follows the
// registry -- elements c, n, o, ne, s, ar, mg, fe, si, cl, ca with a
// positive abundance, stages 1..nstage-1 -- and indexes the rate cache, the
// Gamma/heating outputs and the cooling sums.  Threshold order (k) is the
// stable sort by E_th of species_setup (species_mod.f90:207-225): a packet
// of energy E sees the prefix k < nm(E), so the packet cross sections, the
// per-leaf opacity weights and the path tallies use it.
#pragma once
#include <string>
#include <vector>

#include "mochii_gpu.h"
#include "thermal.h"

namespace mochii {

constexpr int kMaxEl = 11, kMaxSt = 6, kMaxTr = 64;   // species_mod.f90:53, define.f90:80

struct MetalEl {          // one element
    int Z, nstage, tr0, st0;   // first transition / stage in element order
    int kind;                  // 1 = C, 2 = O (H-impact fine-structure lines), 0 otherwise
    double abund;
};

struct MetalTr {          // one transition, element order
    int ie, it, flat;          // element (0-based), stage (1-based), threshold-order index
    int cxi_form, cxr_form, ndr, has_dr2, has_rr2;
    double eth, cidr;          // cidr: ci_dere_ratio(Z, it)
    double ci[5], rr[6], dr_c[9], dr_e[9], dr2[4], rr2[2], cxi[6], cxr[6];
};

struct MetalStage {       // one (element, stage), element order
    int has_cool, nterm, table;   // table: index of the n-level table, -1 = fit only
    double A[kMaxFitTerms], Ti[kMaxFitTerms];
};

struct SpeciesHost {
    std::vector<MetalEl> el;
    std::vector<MetalTr> tr;          // element order
    std::vector<MetalStage> st;       // element order
    std::vector<double> photo;        // threshold order: 8 per transition
    std::vector<int> form;            // threshold order: 1 VFKY96, 2 VY95
    std::vector<double> eth_flat;     // threshold order
    std::vector<double> lamref, Ssup; // n-level tables: ntab x kNlNT, ntab x kNlNT x kNlNNE
    int ntab = 0;
    std::vector<double> thresholds() const;   // element order (main.f90:65-82)
    // energy-moment tally (metal_tally = 'moments'): bin edges and the
    // Chebyshev coefficients of sigma_k/E and sigma_k (1 - E_th,k/E) per bin
    std::vector<double> medge, mcoef;
    std::vector<int> mb0;             // threshold order: first bin where the transition is active
};

constexpr int kMomDeg = 6;            // Chebyshev moments per bin (degree 5)
constexpr double kMomTol = 2.0e-7;    // interpolation error bound per bin, relative to the bin's peak

// Moment bins over [emin, emax]: the H/He and metal thresholds inside are
// edges, each sub-range is split log-uniformly with ln(hi/lo) <= 0.04 per
// bin, and in every bin both rate integrands of every active transition are
// interpolated at the kMomDeg Chebyshev nodes (1e-18 cm^2 units).  A bin
// whose interpolant misses any integrand by more than kMomTol of that
// integrand's peak over the bin (checked at 33 points) is halved in ln E.
void species_moment_tables(SpeciesHost& s, double emin, double emax);

// Device copy: registry tables plus the per-leaf metal arrays.
struct MetalDev {
    int nel = 0, ntr = 0, nst = 0, ntrp = 0;   // ntrp: ntr padded to a multiple of 4
    const MetalEl* el = nullptr;
    const MetalTr* tr = nullptr;
    const MetalStage* st = nullptr;
    const double* photo = nullptr;
    const int* form = nullptr;
    const double* eth = nullptr;       // threshold order
    const double* lamref = nullptr;
    const double* Ssup = nullptr;
    const double* lnL = nullptr;       // log(lamref * Ssup) per table (0 where not positive)
    double* egam = nullptr;            // nleaf x ntr, element order [s^-1]
    double* eheat = nullptr;           // nleaf x ntr, element order [erg/s]
    void* opac = nullptr;              // nleaf x ntrp (R), threshold order: n_H A_el f_it d2cm 1e-18
    void* raw = nullptr;               // nleaf x ntrp x 2 tallies (FP64 or FP32 pairs), threshold order
    int nmb = 0;                       // moment bins (0: exact tallies)
    const double* medge = nullptr;     // nmb + 1
    const double* mcoef = nullptr;     // (nmb*kMomDeg) x ntrp x 2
    const int* mb0 = nullptr;          // ntr, threshold order
    const int* jof = nullptr;          // ntrp: element-order index of each threshold-order index (-1: padding)
    void* mom = nullptr;               // nleaf x nmb x kMomDeg tallies, or with mom32 nleaf x nmb x 8 floats
    int mom32 = 0;                     // FP32 moments, one 32-byte sector per (leaf, bin): FP32 segments with FP64 tallies
    int raw32 = 0;                     // FP32 exact tallies (same condition): 8 bytes per transition, vector reductions
    // T table of the rate coefficients (thermal solve): ln of collisional
    // ionisation, recombination, CX ionisation, CX recombination per
    // transition on tnt nodes uniform in ln T from tu0 by tdu,
    // ttab[(j * 4 + c) * tnt + i]; tnt == 0: exact evaluation only
    const double* ttab = nullptr;
    const double* ctab = nullptr;      // nst x tnt: ln of each stage's line-cooling fit at the same nodes
    int tnt = 0;
    double tu0 = 0.0, tdu = 0.0;
};

bool species_build(const mochii_params& p, SpeciesHost& s, std::string* err);
// n-level (T, n_e) suppression table of one atom file (nlevel_cooling_mod.f90:104-163);
// false when the file is absent.
bool nlevel_table_build(const std::string& path, std::vector<double>& lamref, std::vector<double>& Ssup);

}  // namespace mochii
