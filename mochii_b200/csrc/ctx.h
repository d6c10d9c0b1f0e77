// Library context: everything one nebula needs on one device.  No global
// state, so several contexts (nebulae) can coexist in a process.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "band.h"
#include "diffuse.h"
#include "dust.h"
#include "mochii_gpu.h"
#include "octree.h"
#include "qmc.cuh"
#include "species.h"
#include "thermal.h"

namespace mochii {

// Device-resident layout (structure of arrays over leaves, raster order for
// the Cartesian grid, leaf index = ix + nx*(iy + ny*iz)):
//   state   FP64: nH, xHI, xHeI, xHeII, ne, Te                 (6 x nleaf)
//   columns per-leaf absorber columns n_i * distance2cm * 1e-18 [1/(1e-18 cm^2)
//           per code length], nabs = 1 (H I) or 4 (H I, He I, He II, pad);
//           FP64 or FP32 by the transport precision
//   tally   per-leaf rate sums, ntally = 2 (Gamma_HI, H_HI) or 6 (+He I, He II);
//           FP64 or (hi, lo) FP32 pairs
//   jt      per-leaf diagnostic spectrum, nnu_band bins per leaf, same type
//   rates   FP64 Gamma/heat, 6 x nleaf (gamma_HI..heat_HeII)
struct DeviceTables {
    double* tab_e = nullptr;   // concatenated sampler knots of all components
    double* tab_f = nullptr;
    double* tab_c = nullptr;
    int* tab_off = nullptr;    // ncomp + 1 offsets
    double* comp = nullptr;    // per component: cdf, x, y, z
    double* eedge = nullptr;   // nnu_band + 1
    QmcTables* qmc = nullptr;
};

struct Grid {
    int nx = 0, ny = 0, nz = 0;
    long long nleaf = 0;
    double xmin = 0, xmax = 0, ymin = 0, ymax = 0, zmin = 0, zmax = 0, dcell = 0;
};

struct TransportWork {
    double* ledger = nullptr;              // per block: emitted, absorbed, escaped
    unsigned long long* counters = nullptr;  // segments, walk kills
    int ledger_blocks = 0;
};

// Peel-off imaging (par%ion_peel; ion_peel_mod.f90): the observers on the
// device and the images the imaging pass accumulates.
struct PeelDev {
    int nobs = 0, nchan = 1, nxim = 0, nyim = 0, direc0 = 0;
    const double* obs = nullptr;     // kPeelObs doubles per observer (see peel.cpp)
    const int* chan = nullptr;       // image channel of each band bin
    double* img_dir = nullptr;       // (nobs, nchan, nyim, nxim): erg/s per code length^2
    double* img_sca = nullptr;
    double* img_dir0 = nullptr;      // save_direc0 only
};
constexpr int kPeelObs = 18;         // x, y, z, alpha, beta, gamma, distance, dxim, dyim, R (row-major)

// Per-packet launch records of one chunk (see transport.cu).
struct RecordBuffers {
    double* tm = nullptr;
    double* td = nullptr;
    int* cell = nullptr;
    int* bits = nullptr;
    void* sig = nullptr;
    void* coef = nullptr;
    double* E = nullptr;      // metals: packet energy
    void* msig = nullptr;     // metals: ntrp x cap cross sections
    void* dsc = nullptr;      // scattering: 2 x cap (dust scattering coefficient, <cos>)
    double* p0 = nullptr;     // scattering on the Cartesian grid: start point and direction, 6 x cap
    long long cap = 0;
    // packet_order 'direction': keys, the walk order, and the sort's buffers
    unsigned* key = nullptr;
    unsigned* key_sorted = nullptr;
    int* seq = nullptr;       // 0 .. cap-1
    int* perm = nullptr;
    void* sort_tmp = nullptr;
    size_t sort_bytes = 0;
};

// Launch shapes chosen by the autotuner (tune.cu) or set by hand.
struct Tuning {
    int lookahead = 2;            // walk look-ahead depth 0..2
    int walk_blocks_per_sm = 8;   // persistent walk grid = SMs x this, 128-thread blocks
    bool tuned = false;
    double best_ms = 0.0;
    int lane_threads = 0;         // per-lane thermal solve: lanes per block (0: the most the cache fits)
    double thermal_ms = 0.0;
};

struct BalanceWork {
    double* partial = nullptr;   // per block: max_dx, max_dte, sum_dxv, sum_xv, sum_dtv, sum_tv
    unsigned long long* counters = nullptr;
    int blocks = 0;
    // the lockstep thermal solve visits leaves sorted by the cascade sums
    // each needed in the previous update, so a warp's leaves need similar work
    unsigned* work = nullptr;         // per leaf: cascade sums of its last solve (clamped to 16 bits)
    unsigned* work_sorted = nullptr;
    int* iota = nullptr;              // 0 .. nleaf-1
    int* order = nullptr;             // leaves by ascending work
    void* sort_tmp = nullptr;
    size_t sort_bytes = 0;
    unsigned long long* next = nullptr;   // the flat / lockstep solves' work counter
    int ls_blocks = 0;                    // the lockstep solve's persistent grid
    // the per-lane solve (metal cache in shared memory): block size, grid, bytes
    int lane_threads = 0, lane_blocks = 0;
    size_t lane_smem = 0;
    bool have_work = false;
};

}  // namespace mochii

struct mochii_ctx {
    mochii_params par;
    mochii::BandSetup band;
    mochii::Grid grid;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evA = nullptr, evB = nullptr;
    bool columns_fresh = false;   // absorber columns match the state
    bool fp32 = false;
    bool tally64 = true;          // FP64 tallies (always with FP64 segments)
    int nabs = 1, ntally = 2, nnu = 0;
    // device memory
    double *nH = nullptr, *xHI = nullptr, *xHeI = nullptr, *xHeII = nullptr, *ne = nullptr, *Te = nullptr;
    void* col = nullptr;
    void* tally = nullptr;
    void* jt = nullptr;
    double* rates = nullptr;
    mochii::DeviceTables tab;
    mochii::TransportWork tw;
    mochii::RecordBuffers rec;
    mochii::Tuning tune;
    mochii::ThermalDev th;          // thermal tables (solve_te)
    mochii::DiffuseBuffers dif;     // diffuse field (diffuse_field)
    mochii::MetalDev metal;         // trace metals (use_metals); metal.ntr == 0 without
    mochii::OctDev oct;             // grid_type = 'amr'; oct.ncells == 0 on the Cartesian grid
    void* oct_blob = nullptr;       // octree: the one allocation behind oct's pointers
    mochii::DustDev dust;           // ion_add_dust grain optics; dust.n == 0 without
    mochii::DustHost dust_host;
    double* dust_blob = nullptr;    // the allocation behind dust's tables
    double* rhokap = nullptr;       // ion_add_dust: grey dust opacity per leaf [1/code length]
    double* ttab = nullptr;         // metals with solve_te: the T table of the rate coefficients
    double* metal_lnl = nullptr;    // metals: log of the n-level suppression tables
    bool xscore = false;            // dust or FUV path estimators (8 tallies per leaf)
    bool scatter = false;           // ion_dust_scatter: forced first interaction and scattered flights
    std::vector<double> lhalf;      // octree: leaf half widths (host copy for leaf_half)
    double* twarm = nullptr;        // bracketed thermal solve: warm-start T_e per leaf ("T_warm")
    bool twarm_set = false;         // consumed by the next thermal update
    double twarm_fac = 1.05;        // first bracketing step from the warm start (learned: narrower)
    double twarm_gate = 0.0;        // residual gate of a learned warm start (0: none)
    bool twarm_learned = false;     // the warm start came from mochii_mlp_warm_start
    double* twarm_err = nullptr;    // device: sum of ln^2(T_e / T_warm) and its count after a learned start
    double warm_err_ln = 0.0;       // RMS of ln(T_e / T_warm) of the last learned warm start (0: none yet)
    // equilibrium dust temperature (dust_temp_mod.f90), built on first use
    double* tdust = nullptr;        // nleaf T_dust [K]
    double* tdust_tab = nullptr;    // lam_ir | sabs_ir | tgrid | femit
    mochii::DustTempHost tdust_host;
    // plane-parallel slab: the boundary tally of the last pass (jtally_mod.f90:39-86)
    double* slab_iesc = nullptr;    // device: 2 x slab_nmu escaping luminosity, top | bottom [erg/s]
    std::vector<double> slab_host;  // its copy after the pass
    mochii::SpeciesHost species;
    bool thermal_ready = false;
    mochii::BalanceWork bw;
    // bumped by every call that changes a launch parameter or reallocates a
    // buffer a recorded batch graph holds (set_nphotons, set_tuning,
    // autotune, the T_warm buffer); a batch refuses to replay after a change
    uint64_t generation = 0;
    mochii_pass_stats last_pass = {};   // statistics of the last transport pass (the rates file's ledger)
    mochii::PeelDev peel;                 // par%ion_peel: observers and images
    std::vector<double> peel_obs;         // host copy of the observers (kPeelObs each)
    void* peel_blob = nullptr;            // the allocation behind peel's pointers
    bool peel_done = false;               // an imaging pass has filled the images
    bool peeling = false;                 // the pass in progress peels (mochii_transport_pass with_peel)
    std::string last_error;
};
