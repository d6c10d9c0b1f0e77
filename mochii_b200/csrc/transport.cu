// Ionising-band transport pass on the device.
//
// One thread carries one packet at a time (grid-stride over packet
// indices, so the launch set is the global Sobol sequence whatever the
// grid shape): Owen-scrambled Sobol launch (qmc_mod.f90), source-energy
// CDF inversion (energy_sampler_mod.f90:187-238), isotropic point emission
// (ion_band_mod.f90:2232-2247), the packet's cross sections at its exact
// energy (ion_packet_mod.f90:21-53), then the analytic zero-variance edge
// walk through the Cartesian grid by the Amanatides-Woo stepping of
// raytrace_amr.f90:495-592, scoring every segment's expected path
// luminosity into the per-leaf rate tallies (ion_score_mod.f90:137-231) and
// the packet's energy into the emitted/absorbed/escaped ledger
// (ion_score_mod.f90:233-252).
//
// Geometry (positions, tMax/tDelta, face choice) is FP64 and compiled
// without FMA contraction, so leaf sequences equal the reference's FP64
// walk bit for bit.  Opacity, attenuation and tallies run in the
// precision of R: FP64, or FP32 with compensated (hi, lo) tally pairs that
// are summed in FP64 by the rate kernel.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <type_traits>

#include <cub/cub.cuh>

#include "ctx.h"
#include "metals.cuh"
#include "physics.cuh"
#include "qmc.cuh"
#include "records.cuh"
#include "transport.h"

namespace mochii {

namespace {

constexpr int kThreads = 256;

struct PassArgs {
    const QmcTables* qmc;
    const double* tab_e;
    const double* tab_f;
    const double* tab_c;
    const int* tab_off;
    const double* comp;   // ncomp x (cdf, x, y, z)
    const double* eedge;
    const void* col;
    void* tally;
    void* jt;
    double* ledger;
    unsigned long long* counters;
    long long np;
    double Lpacket;
    double org[3];
    double dcell;
    int n[3];
    int ncomp, multi, ndim, nnu;
    int ext_ic, ext_sph;   // the external field's component (-1 none) and entry surface (0 box faces, 1 sphere)
    double ext_rmax;       // the entry sphere's radius (code units)
    double bmin[3], bmax[3];   // the grid box (code units)
    int xyper;             // par%xy_periodic: the walks wrap the x and y faces, z faces are open
    int slab;              // plane-parallel slab illumination (the one component)
    int slab_mode[2];      // per face [top, bottom]: 0 beam, 1 Lambert
    double slab_mu[2], slab_phi[2], slab_ptop;
    int slab_nmu;          // mu bins of the boundary tally
    double* slab_iesc;     // 2 x slab_nmu luminosity escaping the top | bottom face, null: no tally
    MetalDev m;          // trace metals; m.ntr == 0 without
    int metal_abs;       // par%ion_metal_abs
    OctDev oct;          // octree grid; oct.ncells == 0 on the Cartesian grid
    DustDev dust;        // grain optics (ion_add_dust); dust.n == 0 without
    const double* rhokap;   // grey dust opacity per leaf (scattered flights' albedo)
    PeelDev peel;        // peel-off observers and images
    int peeling;         // this pass is the imaging pass (with_peel)
    int xs;              // dust or FUV path estimators (8 tallies per leaf)
    int scatter;         // ion_dust_scatter
    double eion_min;
    unsigned long long seed;   // par%iseed: key of the scattered flights' streams
};

// ---- octree geometry (octree_mod.f90) ------------------------------------------
// One 32-byte geometry record (centre, half width) through the read-only path.
__device__ __forceinline__ double4 ld_geo(const double4* p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// amr_find_leaf (:69-93): descent from the root by centre comparisons.  The
// complete top levels (cells below nshared, all internal cells) come from
// the copy staged in shared memory when the caller passes one.
__device__ __forceinline__ int oct_find_leaf(const OctDev& o, double x, double y, double z,
                                             const double4* sgeo = nullptr, const int* schild = nullptr) {
    if (o.car) {   // car_index (octree_mod.f90:185-195) inside the box
        if (x < o.org[0] || x > o.hi[0] || y < o.org[1] || y > o.hi[1] || z < o.org[2] || z > o.hi[2]) return -1;
        const int ix = min(max((int)((x - o.org[0]) / o.dcell), 0), o.n[0] - 1);
        const int iy = min(max((int)((y - o.org[1]) / o.dcell), 0), o.n[1] - 1);
        const int iz = min(max((int)((z - o.org[2]) / o.dcell), 0), o.n[2] - 1);
        return ix + o.n[0] * (iy + o.n[1] * iz);
    }
    const double h = o.half;
    if (x < -h || x > h || y < -h || y > h || z < -h || z > h) return -1;
    int c = 0;
    for (int guard = 0; guard < 64; ++guard) {
        const bool st = sgeo && c < o.nshared;
        if (!st) {
            const int lf = __ldg(o.ileaf + c);
            if (lf >= 0) return lf;
        }
        const double4 g = st ? sgeo[c] : ld_geo(o.geo + c);
        int ioct = 0;
        if (x >= g.x) ioct += 1;
        if (y >= g.y) ioct += 2;
        if (z >= g.z) ioct += 4;
        c = st ? schild[8 * c + ioct] : __ldg(o.children + 8 * c + ioct);
        if (c < 0) return -1;
    }
    return -1;
}

// Stage the complete top levels (geometry and children) in shared memory.
__device__ __forceinline__ void oct_stage(const OctDev& o, double4* sgeo, int* schild) {
    for (int i = threadIdx.x; i < o.nshared; i += blockDim.x) sgeo[i] = o.geo[i];
    for (int i = threadIdx.x; i < 8 * o.nshared; i += blockDim.x) schild[i] = o.children[i];
}

// amr_cell_exit (:308-340): distance to the nearest face of the cell and the
// face (0 +x, 1 -x, 2 +y, 3 -y, 4 +z, 5 -z); minloc over the six candidate
// times in that order (first minimum on ties), a non-moving axis giving huge.
__device__ __forceinline__ double oct_cell_exit(const double4 g, double x, double y, double z, double kx, double ky,
                                                double kz, int* face) {
    double t0 = kHugest, t1 = kHugest, t2 = kHugest, t3 = kHugest, t4 = kHugest, t5 = kHugest;
    if (kx > 0.0) t0 = (g.x + g.w - x) / kx; else if (kx < 0.0) t1 = (g.x - g.w - x) / kx;
    if (ky > 0.0) t2 = (g.y + g.w - y) / ky; else if (ky < 0.0) t3 = (g.y - g.w - y) / ky;
    if (kz > 0.0) t4 = (g.z + g.w - z) / kz; else if (kz < 0.0) t5 = (g.z - g.w - z) / kz;
    double t = t0;
    int f = 0;
    if (t1 < t) { t = t1; f = 1; }
    if (t2 < t) { t = t2; f = 2; }
    if (t3 < t) { t = t3; f = 3; }
    if (t4 < t) { t = t4; f = 4; }
    if (t5 < t) { t = t5; f = 5; }
    *face = f;
    return t;
}

// amr_next_leaf (:499-537) from a leaf: the leaf across the face when the
// face neighbour is one, else descent from the neighbour by the two
// tangential coordinates with the face-normal octant bit set by the face.
__device__ __forceinline__ int oct_next_leaf(const OctDev& o, int il, int face, double x, double y, double z) {
    const int nx = __ldg(o.lnext + 8 * il + face);
    if (nx >= -1) return nx;
    int n = -2 - nx;
    for (int guard = 0; guard < 64; ++guard) {
        const double4 g = ld_geo(o.geo + n);
        int ioct = 0;
        if (face == 0 || face == 1) {
            ioct = face == 1 ? 1 : 0;
            if (y >= g.y) ioct += 2;
            if (z >= g.z) ioct += 4;
        } else if (face == 2 || face == 3) {
            if (x >= g.x) ioct += 1;
            ioct += face == 3 ? 2 : 0;
            if (z >= g.z) ioct += 4;
        } else {
            if (x >= g.x) ioct += 1;
            if (y >= g.y) ioct += 2;
            ioct += face == 5 ? 4 : 0;
        }
        const int ch = __ldg(o.children + 8 * n + ioct);
        if (ch < 0) return -1;   // no child there: the walk ends
        const int lf = __ldg(o.ileaf + ch);
        if (lf >= 0) return lf;
        n = ch;
    }
    return -1;
}

// sample_energy_cdf, energy_sampler_mod.f90:187-238.  The bracket search and
// the exact inverse of the linear density follow the same FP64 operation
// sequence as the host restatement, so energies are bit-identical to it.
__device__ double sample_energy(const double* __restrict__ e, const double* __restrict__ f,
                                const double* __restrict__ c, int n, double u) {
    const double q = fmin(fmax(u, 0.0), 1.0);
    if (q <= 0.0) return e[0];
    if (q >= 1.0) return e[n - 1];
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi + 2) / 2 - 1;
        if (__ldg(c + mid) <= q) lo = mid; else hi = mid;
    }
    const double clo = __ldg(c + lo), chi = __ldg(c + hi);
    const double area = chi - clo;
    const double elo = __ldg(e + lo), ehi = __ldg(e + hi);
    if (area <= 0.0) return ehi;
    const double dx = ehi - elo;
    const double y0 = __ldg(f + lo), y1 = __ldg(f + hi);
    const double a = (q - clo) / area * (0.5 * (y0 + y1) * dx);
    const double slope = (y1 - y0) / dx;
    const double sc = fmax(fmax(fabs(y0), fabs(y1)), kTinest);
    double off;
    if (fabs(slope * dx) <= 64.0 * 2.220446049250313e-16 * sc)
        off = y0 > 0.0 ? a / y0 : 0.0;
    else
        off = 2.0 * a / (y0 + sqrt(fmax(0.0, y0 * y0 + 2.0 * slope * a)));
    return elo + fmin(fmax(off, 0.0), dx);
}

// ion_bin_of with include_fuv (ion_band_mod.f90:624-646), 0-based bin.
__device__ int bin_of(const double* __restrict__ edge, int nnu, double eph) {
    int lo = 1, hi = nnu;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (__ldg(edge + mid - 1) <= eph) lo = mid; else hi = mid - 1;
    }
    return min(max(lo, 1), nnu) - 1;
}

// Compensated FP32 accumulation: the atomic returns the old value, the
// rounding error of old + v is recovered exactly (Knuth TwoSum, valid for a
// round-to-nearest add) and accumulated in the low word.
__device__ __forceinline__ void tally_add(float2* p, float v) {
    const float old = atomicAdd(&p->x, v);
    const float s = old + v;
    const float bp = s - old;
    const float err = (old - (s - bp)) + (v - bp);
    if (err != 0.0f) atomicAdd(&p->y, err);
}
__device__ __forceinline__ void tally_add(double* p, double v) { atomicAdd(p, v); }

// Path weight of one segment of optical depth ks > 0 and the attenuation
// after it: (expo - expo e^-ks) / kap (raytrace_amr.f90:462).  In FP32 the
// difference of two attenuations keeps only about ulp/ks of relative
// precision on a thin segment, so below ks = 1/4 the absorbed fraction comes
// from expm1f; FP64 keeps the reference's own difference.
__device__ __forceinline__ float segment_weight(float& expo, float ks, float kap) {
    const float eo = expo * expf(-ks);
    const float w = (ks < 0.25f ? -expo * expm1f(-ks) : expo - eo) / kap;
    expo = eo;
    return w;
}
__device__ __forceinline__ double segment_weight(double& expo, double ks, double kap) {
    const double eo = expo * exp(-ks);
    const double w = (expo - eo) / kap;
    expo = eo;
    return w;
}


template <typename R, int NABS>
__device__ __forceinline__ R opacity(const void* col, long long il, R s0, R s1, R s2) {
    if constexpr (NABS == 1) {
        const R c = __ldg(static_cast<const R*>(col) + il);
        return c * s0;
    } else if constexpr (sizeof(R) == 4) {
        const float4 c = __ldg(static_cast<const float4*>(col) + il);
        return c.x * s0 + (c.y * s1 + c.z * s2);
    } else {
        const double2* p = static_cast<const double2*>(col) + 2 * il;
        const double2 c01 = __ldg(p);
        const double c2 = __ldg(reinterpret_cast<const double*>(p + 1));
        return c01.x * s0 + (c01.y * s1 + c2 * s2);
    }
}

// Block reduction of a double in fixed order (deterministic).
__device__ double block_sum(double v, double* sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (t < s) sh[t] = sh[t] + sh[t + s];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// Launch kernel: one thread per packet, no divergence between packets.
// gen_ion_photon_qmc (ion_band_mod.f90:1880-1935) with emit_point_qmc
// (:2232-2247), build_ion_packet_physics (ion_packet_mod.f90:21-53), the
// coefficients of score_ion_path (ion_score_mod.f90:213-221) and dda_init
// (raytrace_amr.f90:495-532).
//
// AMR: the octree variant stages the complete top levels of the tree in
// shared memory for the start-leaf search.
// emit_external_rec_qmc (ion_band_mod.f90:2253-2323): the isotropic
// external field entering the box: an area-weighted face (u_face), a
// Lambert incidence about its inward normal (mu = sqrt(u_mu), azimuth
// 2 pi u_phi), the entry point uniform on the face (u_c1, u_c2), nudged
// 1e-6 of the smallest extent inside.
__device__ void emit_external_rec(const PassArgs& a, double u_mu, double u_phi, double u_face, double u_c1,
                                  double u_c2, double pos[3], double kk[3], int* face_out = nullptr) {
    const double xr = a.bmax[0] - a.bmin[0], yr = a.bmax[1] - a.bmin[1], zr = a.bmax[2] - a.bmin[2];
    const double nudge = 1.0e-6 * fmin(xr, fmin(yr, zr));
    double fcum[6];
    fcum[0] = yr * zr;
    fcum[1] = fcum[0] + yr * zr;
    fcum[2] = fcum[1] + zr * xr;
    fcum[3] = fcum[2] + zr * xr;
    fcum[4] = fcum[3] + xr * yr;
    fcum[5] = fcum[4] + xr * yr;
    const double fpick = u_face * fcum[5];
    int f = 5;
    for (int k = 0; k < 6; ++k)
        if (fpick <= fcum[k]) { f = k; break; }
    const double mu = sqrt(u_mu), sinm = sqrt(1.0 - mu * mu);
    double sphi, cphi;
    sincos(kTwoPi * u_phi, &sphi, &cphi);
    const int ax = f >> 1;                        // the face's axis: x, y, z
    const double sgn = (f & 1) ? 1.0 : -1.0;      // inward normal along it: -1 on the + face
    const int a1 = ax == 0 ? 1 : 0, a2 = ax == 2 ? 1 : 2;   // the in-face coordinates, in order
    pos[ax] = (f & 1) ? a.bmin[ax] + nudge : a.bmax[ax] - nudge;
    pos[a1] = a.bmin[a1] + (a.bmax[a1] - a.bmin[a1]) * u_c1;
    pos[a2] = a.bmin[a2] + (a.bmax[a2] - a.bmin[a2]) * u_c2;
    kk[ax] = sgn * mu;
    kk[a1] = sinm * cphi;
    kk[a2] = sinm * sphi;
    if (face_out) *face_out = f;
}

// emit_external_sph_qmc (:2328-2361) with ortho_frame (:2368-2385): the
// entry point uniform on the sphere of radius rmax about the box centre
// (u_cost, u_saz), a Lambert incidence about the inward radial (u_mu,
// u_phi) in a frame completed from the coordinate axis most orthogonal to
// it, the point nudged inside.
__device__ void emit_external_sph(const PassArgs& a, double u_mu, double u_phi, double u_cost, double u_saz,
                                  double pos[3], double kk[3]) {
    const double xc = 0.5 * (a.bmin[0] + a.bmax[0]), yc = 0.5 * (a.bmin[1] + a.bmax[1]);
    const double zc = 0.5 * (a.bmin[2] + a.bmax[2]);
    const double cost = 2.0 * u_cost - 1.0, sint = sqrt(1.0 - cost * cost);
    double sp, cp;
    sincos(kTwoPi * u_saz, &sp, &cp);
    const double rx = sint * cp, ry = sint * sp, rz = cost;
    pos[0] = xc + a.ext_rmax * rx;
    pos[1] = yc + a.ext_rmax * ry;
    pos[2] = zc + a.ext_rmax * rz;
    const double nx = -rx, ny = -ry, nz = -rz;
    double tx, ty, tz;
    if (fabs(nx) <= fabs(ny) && fabs(nx) <= fabs(nz)) { tx = 0.0; ty = nz; tz = -ny; }
    else if (fabs(ny) <= fabs(nz)) { tx = -nz; ty = 0.0; tz = nx; }
    else { tx = ny; ty = -nx; tz = 0.0; }
    const double inv = 1.0 / sqrt(tx * tx + ty * ty + tz * tz);
    tx = tx * inv; ty = ty * inv; tz = tz * inv;
    const double bx = ny * tz - nz * ty, by = nz * tx - nx * tz, bz = nx * ty - ny * tx;
    const double mu = sqrt(u_mu), sinm = sqrt(1.0 - mu * mu);
    double sphi, cphi;
    sincos(kTwoPi * u_phi, &sphi, &cphi);
    kk[0] = -mu * rx + sinm * (cphi * tx + sphi * bx);
    kk[1] = -mu * ry + sinm * (cphi * ty + sphi * by);
    kk[2] = -mu * rz + sinm * (cphi * tz + sphi * bz);
    const double nudge = 1.0e-6 * fmin(a.bmax[0] - a.bmin[0], fmin(a.bmax[1] - a.bmin[1], a.bmax[2] - a.bmin[2]));
    pos[0] = pos[0] - nudge * rx;
    pos[1] = pos[1] - nudge * ry;
    pos[2] = pos[2] - nudge * rz;
}

// emit_slab_qmc (ion_band_mod.f90:2183-2208): the lit z face drawn by its
// share of the entering flux (u_face against the top's), the entry point
// uniform over it (u_c1, u_c2) nudged 1e-6 of the smallest extent inside,
// the direction a beam at the face's incidence and azimuth or a Lambert ray
// (mu = sqrt(u_mu) floored at 1e-6, azimuth 2 pi u_phi) into the slab.
__device__ void emit_slab(const PassArgs& a, double u_face, double u_c1, double u_c2, double u_mu, double u_phi,
                          double pos[3], double kk[3]) {
    const double xr = a.bmax[0] - a.bmin[0], yr = a.bmax[1] - a.bmin[1], zr = a.bmax[2] - a.bmin[2];
    const double nudge = 1.0e-6 * fmin(xr, fmin(yr, zr));
    const int f = u_face > a.slab_ptop ? 1 : 0;   // 0 top (+z), 1 bottom (-z)
    pos[0] = a.bmin[0] + xr * u_c1;
    pos[1] = a.bmin[1] + yr * u_c2;
    pos[2] = f == 0 ? a.bmax[2] - nudge : a.bmin[2] + nudge;
    double mu, ph;
    if (a.slab_mode[f]) {
        mu = fmax(sqrt(u_mu), 1.0e-6);
        ph = kTwoPi * u_phi;
    } else {
        mu = a.slab_mu[f];
        ph = a.slab_phi[f];
    }
    const double sinm = sqrt(fmax(1.0 - mu * mu, 0.0));
    double sp, cp;
    sincos(ph, &sp, &cp);
    kk[0] = sinm * cp;
    kk[1] = sinm * sp;
    kk[2] = f == 0 ? -mu : mu;
}

// The launch of one stellar packet from its uniforms u (gen_ion_photon_qmc,
// ion_band_mod.f90:1880-1935): a single point source reads u1 energy, u2 mu,
// u3 phi; the slab u1 energy, u2 face, u3/u4 the entry point, u5 mu, u6
// phi; every other configuration the superset layout -- u1 component, u2
// energy, u3/u4 angles, u5-u7 the entry surface of an external field.
__device__ __forceinline__ void launch_packet(const PassArgs& a, const double* u, int& ic, double& E, double pos[3],
                                              double kk[3], int* xface = nullptr) {
    ic = 0;
    if (xface) *xface = -1;
    double umu, uphi, ue;
    if (a.slab) {
        const int t0 = a.tab_off[0], t1 = a.tab_off[1];
        E = sample_energy(a.tab_e + t0, a.tab_f + t0, a.tab_c + t0, t1 - t0, u[0]);
        emit_slab(a, u[1], u[2], u[3], u[4], u[5], pos, kk);
        return;
    }
    if (a.ndim == 3) {
        ue = u[0]; umu = u[1]; uphi = u[2];
    } else {
        if (a.multi) {
            ic = a.ncomp - 1;
            for (int k = 0; k < a.ncomp; ++k)
                if (u[0] <= a.comp[4 * k]) { ic = k; break; }
        }
        ue = u[1]; umu = u[2]; uphi = u[3];
    }
    const int t0 = a.tab_off[ic], t1 = a.tab_off[ic + 1];
    E = sample_energy(a.tab_e + t0, a.tab_f + t0, a.tab_c + t0, t1 - t0, ue);
    if (ic == a.ext_ic) {
        if (a.ext_sph) emit_external_sph(a, u[2], u[3], u[4], u[5], pos, kk);
        else emit_external_rec(a, u[2], u[3], u[4], u[5], u[6], pos, kk, xface);
        if (xface && a.ext_sph) *xface = 6;
    } else {   // emit_point_qmc (:2232-2247)
        pos[0] = a.comp[4 * ic + 1]; pos[1] = a.comp[4 * ic + 2]; pos[2] = a.comp[4 * ic + 3];
        const double cost = 2.0 * umu - 1.0;
        const double sint = sqrt(1.0 - cost * cost);
        double sphi, cphi;
        sincos(kTwoPi * uphi, &sphi, &cphi);
        kk[0] = sint * cphi; kk[1] = sint * sphi; kk[2] = cost;
    }
}

template <typename R, bool AMR>
__global__ void __launch_bounds__(kThreads) k_launch(const PassArgs a, PacketRecords rec, long long ip0, long long n) {
    __shared__ QmcTables sq;
    __shared__ double4 sgeo[AMR ? kOctShared : 1];
    __shared__ int schild[AMR ? 8 * kOctShared : 1];
    if constexpr (AMR) oct_stage(a.oct, sgeo, schild);
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(a.qmc);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&sq);
        for (int i = threadIdx.x; i < (int)(sizeof(QmcTables) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // packet_order 'coherent': record i is the chunk's packet rec.order[i]
    const long long ip = ip0 + (rec.order ? (long long)rec.order[i] : i);
    double u[7];
    for (int d = 0; d < a.ndim; ++d) u[d] = qmc_uniform(sq, (uint64_t)ip, d, 0);
    int ic, xface;
    double E, pos[3], kk[3];
    launch_packet(a, u, ic, E, pos, kk, &xface);
    const int inu = bin_of(a.eedge, a.nnu, E);
    if constexpr (AMR)   // emit_point_qmc: photon%icell_amr = amr_find_leaf (ion_band_mod.f90:2245)
        write_record_amr<R>(rec, i, pos, kk, E, inu, oct_find_leaf(a.oct, pos[0], pos[1], pos[2], sgeo, schild));
    else
        write_record<R>(rec, i, pos, kk, E, inu, a.org, a.dcell, a.n);
    if (xface >= 0) rec.bits[i] |= kExternalBit | (xface << kExternalFaceShift);   // photon%from_external
    if (a.xs) write_grain_record<R>(rec, i, a.dust, a.scatter, a.eion_min, E, pos, kk, AMR ? 0 : 1);
    if (a.m.ntr > 0) write_metal_record<R>(rec, a.m, i, E);
    if (rec.key) rec.key[i] = packet_dir_key(ic, kk);
}

// Walk-order keys of packet_order 'coherent' for packets ip0 .. ip0+n-1 of
// the stellar stream: the launch uniforms of gen_ion_photon_qmc
// (ion_band_mod.f90:1880-1935) reduced to coherent_key.
__global__ void __launch_bounds__(kThreads) k_coherent_keys(const PassArgs a, long long ip0, long long n,
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
    int ic = 0;
    double ue, umu, uphi;
    if (a.ndim == 3) {
        ue = qmc_uniform(sq, ip, 0, 0);
        umu = qmc_uniform(sq, ip, 1, 0);
        uphi = qmc_uniform(sq, ip, 2, 0);
    } else {
        if (a.multi) {
            const double u0 = qmc_uniform(sq, ip, 0, 0);
            ic = a.ncomp - 1;
            for (int k = 0; k < a.ncomp; ++k)
                if (u0 <= a.comp[4 * k]) { ic = k; break; }
        }
        ue = qmc_uniform(sq, ip, 1, 0);
        umu = qmc_uniform(sq, ip, 2, 0);
        uphi = qmc_uniform(sq, ip, 3, 0);
    }
    key[i] = coherent_key(ic, umu, uphi, ue);
}

// Absorber columns of one leaf, loaded ahead of use.
template <typename R, int NABS> struct Col;
// The 4-wide layout's fourth slot is the leaf's rhokap; with X (grains or
// FUV) the packet's dust extinction coefficient s3 multiplies it.
template <typename R> struct Col<R, 1> {
    R c0;
    __device__ __forceinline__ void load(const void* col, int il) { c0 = __ldg(static_cast<const R*>(col) + il); }
    template <int X>
    __device__ __forceinline__ R kappa(R s0, R, R, R) const { return c0 * s0; }
};
template <> struct Col<float, 4> {
    float4 c;
    __device__ __forceinline__ void load(const void* col, int il) { c = __ldg(static_cast<const float4*>(col) + il); }
    template <int X>
    __device__ __forceinline__ float kappa(float s0, float s1, float s2, float s3) const {
        const float k = c.x * s0 + (c.y * s1 + c.z * s2);
        return X ? k + c.w * s3 : k;
    }
};
template <> struct Col<double, 4> {
    double2 a, b;
    __device__ __forceinline__ void load(const void* col, int il) {
        const double2* p = static_cast<const double2*>(col) + 2 * (long long)il;
        a = __ldg(p);
        b = __ldg(p + 1);
    }
    template <int X>
    __device__ __forceinline__ double kappa(double s0, double s1, double s2, double s3) const {
        const double k = a.x * s0 + (a.y * s1 + b.x * s2);
        return X ? k + b.y * s3 : k;
    }
};

// Amanatides-Woo cell stepper (raytrace_amr.f90:553-590): emits the current
// cell and its segment length, then steps to the neighbour across the
// nearest face (minloc first-minimum tie rule).  Pure FP64 geometry, so it
// runs ahead of the opacity work and the column loads of upcoming cells are
// in flight while the current cell is scored.
// per: xy-periodic (raytrace_amr.f90:575-582): a step out of an x or y face
// re-enters at the opposite one (the uniform grid keeps tMax and tDelta), so
// only the z faces end the walk.
struct Stepper {
    double t0, t1, t2, d0, d1, d2, t_cur;
    int ix, iy, iz, sx, sy, sz;
    int per = 0;
    __device__ __forceinline__ bool emit(int nx, int ny, int nz, int* il, double* seg) {
        *il = ix + nx * (iy + ny * iz);
        int ax = 0;
        double tm = t0;
        if (t1 < tm) { ax = 1; tm = t1; }
        if (t2 < tm) { ax = 2; tm = t2; }
        *seg = tm - t_cur;
        t_cur = tm;
        t0 = ax == 0 ? t0 + d0 : t0;
        t1 = ax == 1 ? t1 + d1 : t1;
        t2 = ax == 2 ? t2 + d2 : t2;
        ix += ax == 0 ? sx : 0;
        iy += ax == 1 ? sy : 0;
        iz += ax == 2 ? sz : 0;
        if (per) {
            ix = ix < 0 ? nx - 1 : (ix >= nx ? 0 : ix);
            iy = iy < 0 ? ny - 1 : (iy >= ny ? 0 : iy);
        }
        return ix >= 0 && ix < nx && iy >= 0 && iy < ny && iz >= 0 && iz < nz;   // next cell inside?
    }
};

// slab_bnd_add (jtally_mod.f90:76-86): luminosity leaving a z face into its
// bin of mu = |k_z| (nmu equal bins in (0, 1]), the top face for k_z > 0.
__device__ __forceinline__ void slab_add(const PassArgs& a, double kz, double lum) {
    const int ib = min(max((int)(fabs(kz) * (double)a.slab_nmu), 0), a.slab_nmu - 1);
    atomicAdd(a.slab_iesc + (kz > 0.0 ? 0 : a.slab_nmu) + ib, lum);
}

// slab_wrap_xy (raytrace_amr.f90:330-345): a packet that left an x or y
// face of the box re-enters at the opposite face's exact boundary value.
__device__ __forceinline__ void slab_wrap_xy(const PassArgs& a, int face, double& x, double& y) {
    if (face == 0) x = a.bmin[0];
    else if (face == 1) x = a.bmax[0];
    else if (face == 2) y = a.bmin[1];
    else if (face == 3) y = a.bmax[1];
}

// H/He part of score_ion_path (ion_score_mod.f90:137-231): the rate tallies
// of the leaf and its diagnostic spectrum bin.
//
// With grains or FUV (NT = 8) the last two tallies are dust_abs_path (w x the
// dust absorption coefficient) and fuv_field_path (w for E < eion_min,
// ion_score_mod.f90:163-166,206-209); a zero coefficient skips its update.
template <typename T, typename R, int NT>
__device__ __forceinline__ void score_hhe(T* tal, T* jt, int il, int nnu, int inu, R w, const R* cf) {
    T* tl = tal + (long long)il * NT;
#pragma unroll
    for (int k = 0; k < (NT < 6 ? NT : 6); ++k) tally_add(tl + k, w * cf[k]);
#pragma unroll
    for (int k = 6; k < NT; ++k)
        if (cf[k] != (R)0) tally_add(tl + k, w * cf[k]);
    tally_add(jt + (long long)il * nnu + inu, w);
}

// The trace-metal state of one packet in the walk.  The packet's
// active-prefix cross sections sigma_k sit in dynamic shared memory
// ([k][thread], ntrp x blockDim of R); per segment the leaf's opacity weights
// add sum_k w_k sigma_k to the absorption (species_cached_opacity,
// species_mod.f90:291-303).  The path estimators of species_rate_path_score
// (:329-343) are either scored directly, two tallies per active transition
// (MET = 1, with the heating coefficients sigma_k (1 - E_th,k/E) in a second
// shared array), or as the kMomDeg Chebyshev moments of the packet energy in
// its moment bin (MET = 2), which the rate kernel contracts with the
// tabulated integrands.
template <typename R, int MET>
struct MetalPacket {
    int nm = 0, mb = 0;
    R invE = (R)0;
    R phi[MET == 2 ? kMomDeg : 1];
    __device__ __forceinline__ void setup(const MetalDev& m, const PacketRecords& rec, long long i, R* msg, R* mhc) {
        const int tb = blockDim.x, tx = threadIdx.x;
        const long long c = rec.cap;
        const double E = rec.E[i];
        nm = metal_nactive(m, E);
        invE = (R)(1.0 / E);
        const R* ms = static_cast<const R*>(rec.msig);
        for (int k = 0; k < nm; ++k) {
            const R sk = ms[k * c + i];
            msg[k * tb + tx] = sk;
            if constexpr (MET == 1) mhc[k * tb + tx] = (R)((double)sk * fmax(1.0 - __ldg(m.eth + k) / E, 0.0));
        }
        if constexpr (MET == 2) {   // moment bin and the Chebyshev values T_0..T_5 of E in it
            int lo = 0, hi = m.nmb - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(m.medge + mid) <= E) lo = mid; else hi = mid - 1;
            }
            mb = lo;
            const double e0 = __ldg(m.medge + mb), e1 = __ldg(m.medge + mb + 1);
            const double t = fmin(fmax((2.0 * E - (e0 + e1)) / (e1 - e0), -1.0), 1.0);
            double tm1 = 1.0, tm = t;
            phi[0] = (R)1;
            phi[1] = (R)t;
#pragma unroll
            for (int q = 2; q < kMomDeg; ++q) {
                const double tn = 2.0 * t * tm - tm1;
                phi[q] = (R)tn;
                tm1 = tm;
                tm = tn;
            }
        }
    }
    __device__ __forceinline__ R kappa(const MetalDev& m, int il, const R* msg) const {
        const int tb = blockDim.x, tx = threadIdx.x;
        const R* op = static_cast<const R*>(m.opac) + (long long)il * m.ntrp;
        R km = (R)0;
        for (int k = 0; k < nm; ++k) km = km + __ldg(op + k) * msg[k * tb + tx];
        return km;
    }
    template <typename T>
    __device__ __forceinline__ void score(const MetalDev& m, int il, R w, const R* msg, const R* mhc) const {
        const int tb = blockDim.x, tx = threadIdx.x;
        if constexpr (MET == 1) {
            if constexpr (std::is_same<R, float>::value && std::is_same<T, double>::value) {
                if (m.raw32) {   // FP32 exact tallies: two transitions per vector reduction
                    float* rw = static_cast<float*>(m.raw) + (long long)il * m.ntrp * 2;
                    const R wi = w * invE;
                    int k = 0;
                    for (; k + 1 < nm; k += 2)
                        asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(rw + 2 * k),
                                     "f"(wi * msg[k * tb + tx]), "f"(w * mhc[k * tb + tx]),
                                     "f"(wi * msg[(k + 1) * tb + tx]), "f"(w * mhc[(k + 1) * tb + tx])
                                     : "memory");
                    if (k < nm)
                        asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(rw + 2 * k), "f"(wi * msg[k * tb + tx]),
                                     "f"(w * mhc[k * tb + tx])
                                     : "memory");
                    return;
                }
            }
            T* rw = static_cast<T*>(m.raw) + (long long)il * m.ntrp * 2;
            const R wi = w * invE;
            for (int k = 0; k < nm; ++k) {
                tally_add(rw + 2 * k, wi * msg[k * tb + tx]);
                tally_add(rw + 2 * k + 1, w * mhc[k * tb + tx]);
            }
        } else if constexpr (MET == 2) {
            if constexpr (std::is_same<R, float>::value && std::is_same<T, double>::value) {
                if (m.mom32) {   // FP32 moments: one sector, two vector reductions
                    float* mt = static_cast<float*>(m.mom) + ((long long)il * m.nmb + mb) * 8;
                    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(mt), "f"(w * phi[0]),
                                 "f"(w * phi[1]), "f"(w * phi[2]), "f"(w * phi[3])
                                 : "memory");
                    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(mt + 4), "f"(w * phi[4]), "f"(w * phi[5])
                                 : "memory");
                    return;
                }
            }
            T* mt = static_cast<T*>(m.mom) + ((long long)il * m.nmb + mb) * kMomDeg;
#pragma unroll
            for (int q = 0; q < kMomDeg; ++q) tally_add(mt + q, w * phi[q]);
        }
    }
};

// Per-block end of a walk kernel: the energy ledger (ion_score_energy_packet,
// ion_score_mod.f90:233-252) summed per block, and the counters.
template <bool METAL>
__device__ __forceinline__ void walk_epilogue(const PassArgs& a, double emitted, double absorbed, double escaped,
                                              unsigned long long nseg, unsigned long long kills,
                                              unsigned long long nact, unsigned long long nscat, int accumulate,
                                              double* sh) {
    const double e0 = block_sum(emitted, sh);
    const double e1 = block_sum(absorbed, sh);
    const double e2 = block_sum(escaped, sh);
    if (threadIdx.x == 0) {
        double* L = a.ledger + 3 * blockIdx.x;
        if (accumulate) {
            L[0] += e0; L[1] += e1; L[2] += e2;
        } else {
            L[0] = e0; L[1] = e1; L[2] = e2;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        nseg += __shfl_down_sync(0xffffffffu, nseg, o);
        kills += __shfl_down_sync(0xffffffffu, kills, o);
        nscat += __shfl_down_sync(0xffffffffu, nscat, o);
        if (METAL) nact += __shfl_down_sync(0xffffffffu, nact, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (nseg) atomicAdd(a.counters + 0, nseg);
        if (kills) atomicAdd(a.counters + 1, kills);
        if (METAL && nact) atomicAdd(a.counters + 2, nact);
        if (nscat) atomicAdd(a.counters + 3, nscat);
    }
}

// ---- scattered flights (transport_ion_packet, raytrace_amr.f90:249-323) -------
constexpr int kMaxScatterings = 100000;   // a bound on scatterings per packet; the reference relies on the roulette

// raytrace_ion_to_tau_amr (raytrace_amr.f90:348-420) on the octree and
// raytrace_ion_to_tau_car (:594-676) on the Cartesian grid: from (x, y, z)
// along k to optical depth tau_in (extinction kappa_at(leaf)); scattered
// flights score every segment with wgt x length (score_at).  Returns whether
// the packet is still inside; then (x, y, z) is the interaction point and il
// its leaf.
template <bool AMR, typename KapF, typename ScoreF>
__device__ __forceinline__ bool walk_to_tau(const PassArgs& a, double tau_in, bool tally, double wgt, double& x,
                                            double& y, double& z, double kx, double ky, double kz, int& il,
                                            KapF& kappa_at, ScoreF& score_at, unsigned long long& kills) {
    if constexpr (AMR) {
        if (il < 0) il = oct_find_leaf(a.oct, x, y, z);
        if (il < 0) return false;
        double tau = 0.0;
        for (int nstep = 1;; ++nstep) {
            if (nstep > kMaxWalkSteps) { ++kills; return false; }
            int face;
            const double texit = oct_cell_exit(ld_geo(a.oct.lgeo + il), x, y, z, kx, ky, kz, &face);
            const double kap = (double)kappa_at(il);
            if (tau + texit * kap >= tau_in) {
                const double d = kap > 0.0 ? (tau_in - tau) / kap : texit;
                if (tally) score_at(il, wgt * d);
                x = x + d * kx;
                y = y + d * ky;
                z = z + d * kz;
                return true;
            }
            if (tally) score_at(il, wgt * texit);
            tau = tau + texit * kap;
            x = x + texit * kx;
            y = y + texit * ky;
            z = z + texit * kz;
            int nl = oct_next_leaf(a.oct, il, face, x, y, z);
            if (nl < 0 && a.xyper) {   // raytrace_amr.f90:403-406
                slab_wrap_xy(a, face, x, y);
                if (face <= 3) nl = oct_find_leaf(a.oct, x, y, z);
            }
            if (nl < 0) {   // a scattered flight leaving a z face: the slab's reflected / diffuse part (:407-413)
                if (face >= 4 && a.slab_iesc) slab_add(a, kz, wgt * a.Lpacket);
                return false;
            }
            il = nl;
        }
    } else {
        // dda_init (raytrace_amr.f90:495-532) from the point
        const double pos[3] = {x, y, z}, kk[3] = {kx, ky, kz};
        int idx[3], stp[3];
        double tmax[3], tdel[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            idx[k] = min(max((int)((pos[k] - a.org[k]) / a.dcell), 0), a.n[k] - 1);
            if (kk[k] > 0.0) {
                stp[k] = 1; tmax[k] = (a.org[k] + (double)(idx[k] + 1) * a.dcell - pos[k]) / kk[k]; tdel[k] = a.dcell / kk[k];
            } else if (kk[k] < 0.0) {
                stp[k] = -1; tmax[k] = (a.org[k] + (double)idx[k] * a.dcell - pos[k]) / kk[k]; tdel[k] = -a.dcell / kk[k];
            } else {
                stp[k] = 0; tmax[k] = kHugest; tdel[k] = kHugest;
            }
        }
        double tau = 0.0, t_cur = 0.0;
        bool inside = true;
        for (int nstep = 1;; ++nstep) {
            if (nstep > kMaxWalkSteps) { ++kills; inside = false; break; }
            const int c = idx[0] + a.n[0] * (idx[1] + a.n[1] * idx[2]);
            int ax = 0;
            if (tmax[1] < tmax[ax]) ax = 1;
            if (tmax[2] < tmax[ax]) ax = 2;
            const double seg = tmax[ax] - t_cur;
            const double kap = (double)kappa_at(c);
            if (tau + seg * kap >= tau_in) {
                const double d = kap > 0.0 ? (tau_in - tau) / kap : seg;
                if (tally) score_at(c, wgt * d);
                t_cur = t_cur + d;
                break;
            }
            if (tally) score_at(c, wgt * seg);
            tau = tau + seg * kap;
            t_cur = tmax[ax];
            tmax[ax] = tmax[ax] + tdel[ax];
            idx[ax] += stp[ax];
            if (idx[ax] < 0 || idx[ax] >= a.n[ax]) {
                if (a.xyper && ax < 2) {   // raytrace_amr.f90:639-654
                    idx[ax] = idx[ax] < 0 ? a.n[ax] - 1 : 0;
                } else {
                    if (ax == 2 && a.slab_iesc) slab_add(a, kz, wgt * a.Lpacket);   // :655-660
                    inside = false;
                    break;
                }
            }
        }
        x = x + t_cur * kx;
        y = y + t_cur * ky;
        z = z + t_cur * kz;
        if (a.xyper) {   // the unwrapped end point folded back into the box (:666-672)
            const double xr = a.bmax[0] - a.bmin[0], yr = a.bmax[1] - a.bmin[1];
            x = x - floor((x - a.bmin[0]) / xr) * xr;
            y = y - floor((y - a.bmin[1]) / yr) * yr;
        }
        if (inside) il = idx[0] + a.n[0] * (idx[1] + a.n[1] * idx[2]);
        return inside;
    }
}

// ---- peel-off imaging (ion_peel_mod.f90) ---------------------------------------
// Optical depth from (x, y, z) along (kx, ky, kz) to the box edge at the
// packet's energy, no tally (raytrace_ion_tau_only_car / _amr,
// raytrace_amr.f90:678-775): the DDA from the point on the Cartesian grid,
// leaf exits on the octree (starting in leaf il when known); stops at
// tau_huge.  FP64 geometry as the edge walk.
template <bool AMR, typename KapF>
__device__ double tau_to_edge(const PassArgs& a, double x, double y, double z, double kx, double ky, double kz, int il,
                              KapF& kappa_at) {
    double tau = 0.0;
    if constexpr (AMR) {
        if (il < 0) il = oct_find_leaf(a.oct, x, y, z);
        if (il < 0) return 0.0;
        for (int nstep = 1; nstep <= kMaxWalkSteps; ++nstep) {
            int face;
            const double texit = oct_cell_exit(ld_geo(a.oct.lgeo + il), x, y, z, kx, ky, kz, &face);
            tau = tau + (double)kappa_at(il) * texit;
            if (tau >= kTauHuge) break;
            x = x + texit * kx;
            y = y + texit * ky;
            z = z + texit * kz;
            const int nl = oct_next_leaf(a.oct, il, face, x, y, z);
            if (nl < 0) break;
            il = nl;
        }
    } else {
        const double pos[3] = {x, y, z}, kk[3] = {kx, ky, kz};
        int idx[3], stp[3];
        double tmax[3], tdel[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            idx[k] = min(max((int)((pos[k] - a.org[k]) / a.dcell), 0), a.n[k] - 1);
            if (kk[k] > 0.0) {
                stp[k] = 1; tmax[k] = (a.org[k] + (double)(idx[k] + 1) * a.dcell - pos[k]) / kk[k]; tdel[k] = a.dcell / kk[k];
            } else if (kk[k] < 0.0) {
                stp[k] = -1; tmax[k] = (a.org[k] + (double)idx[k] * a.dcell - pos[k]) / kk[k]; tdel[k] = -a.dcell / kk[k];
            } else {
                stp[k] = 0; tmax[k] = kHugest; tdel[k] = kHugest;
            }
        }
        double t_cur = 0.0;
        for (int nstep = 1; nstep <= kMaxWalkSteps; ++nstep) {
            const int c = idx[0] + a.n[0] * (idx[1] + a.n[1] * idx[2]);
            int ax = 0;
            if (tmax[1] < tmax[ax]) ax = 1;
            if (tmax[2] < tmax[ax]) ax = 2;
            tau = tau + (double)kappa_at(c) * (tmax[ax] - t_cur);
            if (tau >= kTauHuge) break;
            t_cur = tmax[ax];
            tmax[ax] = tmax[ax] + tdel[ax];
            idx[ax] += stp[ax];
            if (idx[ax] < 0 || idx[ax] >= a.n[ax]) break;
        }
    }
    return tau;
}

// The observer-frame pixel of direction (kx, ky, kz) for observer o (the
// TAN image plane of ion_peel_direct, 0-based); false outside the image.
__device__ __forceinline__ bool peel_pixel(const PeelDev& p, const double* o, double kx, double ky, double kz, int* ix,
                                           int* iy) {
    const double v0 = o[9] * kx + o[10] * ky + o[11] * kz;
    const double v1 = o[12] * kx + o[13] * ky + o[14] * kz;
    const double v2 = o[15] * kx + o[16] * ky + o[17] * kz;
    constexpr double r2d = 180.0 / kPi;
    *ix = (int)floor(atan2(-v0, v2) * r2d / o[7] + p.nxim / 2.0);
    *iy = (int)floor(atan2(-v1, v2) * r2d / o[8] + p.nyim / 2.0);
    return *ix >= 0 && *ix < p.nxim && *iy >= 0 && *iy < p.nyim;
}

// ion_peel_direct (ion_peel_mod.f90:225-277): the isotropic source's
// wl / (4 pi r^2) e^-tau (wl = packet luminosity x weight) toward every
// observer's pixel, the unattenuated part to the direc0 image.
template <bool AMR, typename KapF>
__device__ void peel_direct(const PassArgs& a, double x, double y, double z, int il, int inu, double wl,
                            KapF& kappa_at, int bits = 0) {
    const PeelDev& p = a.peel;
    const int ch = __ldg(p.chan + inu);
    // an external packet peels max(k_obs . n_in, 0) / pi about the inward
    // normal of its entry surface (ion_peel_mod.f90:254-263): a box face's
    // axis, or toward the sphere's centre
    const bool ext = bits & kExternalBit;
    double nin[3] = {0.0, 0.0, 0.0};
    if (ext) {
        const int f = (bits >> kExternalFaceShift) & 7;
        if (f < 6) {
            nin[f >> 1] = (f & 1) ? 1.0 : -1.0;
        } else {
            const double dx = x - 0.5 * (a.bmin[0] + a.bmax[0]), dy = y - 0.5 * (a.bmin[1] + a.bmax[1]);
            const double dz = z - 0.5 * (a.bmin[2] + a.bmax[2]);
            const double rr = sqrt(dx * dx + dy * dy + dz * dz);
            nin[0] = -dx / rr; nin[1] = -dy / rr; nin[2] = -dz / rr;
        }
    }
    for (int k = 0; k < p.nobs; ++k) {
        const double* o = p.obs + k * kPeelObs;
        double kx = __ldg(o) - x, ky = __ldg(o + 1) - y, kz = __ldg(o + 2) - z;
        const double r2 = kx * kx + ky * ky + kz * kz, r = sqrt(r2);
        kx = kx / r; ky = ky / r; kz = kz / r;
        int ix, iy;
        if (!peel_pixel(p, o, kx, ky, kz, &ix, &iy)) continue;
        const long long pix = ((long long)(k * p.nchan + ch) * p.nyim + iy) * p.nxim + ix;
        double contrib;
        if (ext) {
            const double cos_obs = kx * nin[0] + ky * nin[1] + kz * nin[2];
            if (cos_obs <= 0.0) continue;   // the observer-side surface shows nothing
            contrib = wl * cos_obs / (kPi * r2);
        } else {
            contrib = wl / (4.0 * kPi * r2);
        }
        if (p.direc0) atomicAdd(p.img_dir0 + pix, contrib);
        const double tau = tau_to_edge<AMR>(a, x, y, z, kx, ky, kz, il, kappa_at);
        if (tau > 500.0) continue;
        atomicAdd(p.img_dir + pix, contrib * exp(-tau));
    }
}

// ion_peel_scatter (ion_peel_mod.f90:284-344): at a dust interaction (after
// the albedo weight, before the new direction; (kx, ky, kz) the incident
// direction) the Henyey-Greenstein phase function toward each observer.
template <bool AMR, typename KapF>
__device__ void peel_scatter(const PassArgs& a, double x, double y, double z, int il, double kx, double ky, double kz,
                             double wl, double g, int inu, KapF& kappa_at) {
    const PeelDev& p = a.peel;
    const int ch = __ldg(p.chan + inu);
    const double gg = fmin(fmax(g, -0.9999), 0.9999);
    const double kn2 = kx * kx + ky * ky + kz * kz;
    for (int k = 0; k < p.nobs; ++k) {
        const double* o = p.obs + k * kPeelObs;
        double ox = __ldg(o) - x, oy = __ldg(o + 1) - y, oz = __ldg(o + 2) - z;
        const double r2 = ox * ox + oy * oy + oz * oz, r = sqrt(r2);
        ox = ox / r; oy = oy / r; oz = oz / r;
        int ix, iy;
        if (!peel_pixel(p, o, ox, oy, oz, &ix, &iy)) continue;
        const double tau = tau_to_edge<AMR>(a, x, y, z, ox, oy, oz, il, kappa_at);
        if (tau > 500.0 || kn2 <= 0.0) continue;
        const double cosa = fmin(fmax((kx * ox + ky * oy + kz * oz) / sqrt(kn2), -1.0), 1.0);
        const double dmin = (1.0 - fabs(gg)) * (1.0 - fabs(gg));
        const double den = fmax((1.0 + gg * gg) - 2.0 * gg * cosa, dmin);
        const double phase = (1.0 - gg * gg) / (den * sqrt(den) * 4.0 * kPi);
        const double contrib = wl * phase / r2 * exp(-tau);
        if (!isfinite(contrib)) continue;
        atomicAdd(p.img_sca + ((long long)(k * p.nchan + ch) * p.nyim + iy) * p.nxim + ix, contrib);
    }
}

// The forced first interaction and the scattered flights of one packet
// (transport_ion_packet after its edge walk): weight 1 - e^-tau_edge, the
// albedo weight rhokap s_sca / kappa at each interaction, Russian roulette
// below 1e-4 (survival 0.1), a Henyey-Greenstein direction about the
// current one, an unforced flight to -ln(u).  Draws come from the packet's
// Philox stream in the reference's order.
template <bool AMR, typename KapF, typename ScoreF, typename PeelF>
__device__ __noinline__ void scattered_flights(const PassArgs& a, double x, double y, double z, double kx, double ky,
                                               double kz, int il, double tau_edge, double ssca, double gg,
                                               uint32_t stream, uint64_t packet, KapF kappa_at, ScoreF score_at,
                                               PeelF peel_at, unsigned long long& kills) {
    PacketStream rs;
    rs.init(a.seed, stream, packet);
    const double w1 = 1.0 - exp(-tau_edge);
    double wgt = w1;
    double tau = -log(1.0 - rs.next() * w1);
    bool inside = walk_to_tau<AMR>(a, tau, false, wgt, x, y, z, kx, ky, kz, il, kappa_at, score_at, kills);
    for (int nev = 1; inside; ++nev) {
        if (il < 0) break;
        if (nev > kMaxScatterings) { ++kills; break; }
        const double a_eff = __ldg(a.rhokap + il) * ssca / fmax((double)kappa_at(il), kTinest);
        wgt = wgt * a_eff;
        peel_at(x, y, z, il, kx, ky, kz, wgt);   // the imaging pass (raytrace_amr.f90:280-281)
        if (wgt < 1.0e-4) {
            if (rs.next() > 0.1) break;
            wgt = wgt / 0.1;
        }
        double cost;
        if (fabs(gg) > 1.0e-3) {
            const double q = (1.0 - gg * gg) / (1.0 + gg * (2.0 * rs.next() - 1.0));
            cost = (1.0 + gg * gg - q * q) / (2.0 * gg);
        } else {
            cost = 2.0 * rs.next() - 1.0;
        }
        cost = fmin(fmax(cost, -1.0), 1.0);
        const double sint = sqrt(1.0 - cost * cost);
        const double phi = kTwoPi * rs.next();
        double norm = sqrt(kx * kx + ky * ky + kz * kz);
        if (norm <= 0.0) break;
        kx = kx / norm; ky = ky / norm; kz = kz / norm;
        double ux, uy, uz;
        if (fabs(kz) < 0.99) { ux = -ky; uy = kx; uz = 0.0; }
        else { ux = 0.0; uy = -kz; uz = ky; }
        norm = sqrt(ux * ux + uy * uy + uz * uz);
        ux = ux / norm; uy = uy / norm; uz = uz / norm;
        const double vx = ky * uz - kz * uy, vy = kz * ux - kx * uz, vz = kx * uy - ky * ux;
        double sp, cp;
        sincos(phi, &sp, &cp);
        const double nx = sint * (cp * ux + sp * vx) + cost * kx;
        const double ny = sint * (cp * uy + sp * vy) + cost * ky;
        const double nz = sint * (cp * uz + sp * vz) + cost * kz;
        norm = sqrt(nx * nx + ny * ny + nz * nz);
        kx = nx / norm; ky = ny / norm; kz = nz / norm;
        tau = -log(fmax(rs.next(), kTinest));
        inside = walk_to_tau<AMR>(a, tau, true, wgt, x, y, z, kx, ky, kz, il, kappa_at, score_at, kills);
    }
}

// Walk kernel: raytrace_ion_to_edge_car (raytrace_amr.f90:534-592) for the
// packets of one chunk, grid-stride.  The stepper runs LA cells ahead of the
// scoring: slot 0 is scored now, slots 1..LA have their column loads in
// flight (LA = 0 disables the look-ahead).
//
// MET adds the trace-metal terms (MetalPacket: 1 exact tallies, 2 moments);
// X the grain and FUV terms (NABS = 4) and, with a.scatter, the scattered
// flights after the edge walk.  Packet i of the chunk is packet ip0 + i of
// its stream (0 stellar, 1 diffuse).
template <typename R, int NABS, int LA, int MET, int X, typename T>
__global__ void __launch_bounds__(128) k_walk_edge(const PassArgs a, const PacketRecords rec, long long n,
                                                   int accumulate, long long ip0, int stream) {
    constexpr int NT = X ? 8 : (NABS == 1 ? 2 : 6);
    constexpr bool METAL = MET > 0;
    __shared__ double sh[128];
    extern __shared__ __align__(16) unsigned char dsm[];
    R* const msg = reinterpret_cast<R*>(dsm);                      // sigma_k      [k][thread]
    R* const mhc = msg + (MET == 1 ? a.m.ntrp * blockDim.x : 0);    // sigma_k h_k  [k][thread]
    double emitted = 0.0, absorbed = 0.0, escaped = 0.0;
    unsigned long long nseg = 0, kills = 0, nact = 0, nscat = 0;
    T* tal = static_cast<T*>(a.tally);
    T* jt = static_cast<T*>(a.jt);
    const R* sg = static_cast<const R*>(rec.sig);
    const R* cfp = static_cast<const R*>(rec.coef);
    const long long c = rec.cap;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int nx = a.n[0], ny = a.n[1], nz = a.n[2];
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const long long i = rec.perm ? (long long)rec.perm[j] : j;
        Stepper g;
        g.t0 = rec.tm[i]; g.t1 = rec.tm[c + i]; g.t2 = rec.tm[2 * c + i];
        g.d0 = rec.td[i]; g.d1 = rec.td[c + i]; g.d2 = rec.td[2 * c + i];
        g.t_cur = 0.0;
        g.per = a.xyper;
        const int cell = rec.cell[i], bits = rec.bits[i];
        g.ix = cell & 1023; g.iy = (cell >> 10) & 1023; g.iz = (cell >> 20) & 1023;
        g.sx = ((bits >> 16) & 3) - 1; g.sy = ((bits >> 18) & 3) - 1; g.sz = ((bits >> 20) & 3) - 1;
        const int inu = bits & 0xFFFF;
        const R s0 = sg[i];
        const R s1 = NABS == 1 ? (R)0 : sg[c + i];
        const R s2 = NABS == 1 ? (R)0 : sg[2 * c + i];
        const R s3 = X ? sg[3 * c + i] : (R)0;
        R cf[NT];
#pragma unroll
        for (int k = 0; k < NT; ++k) cf[k] = cfp[k * c + i];
        MetalPacket<R, MET> mp;
        if constexpr (METAL) mp.setup(a.m, rec, i, msg, mhc);
        if (a.peeling) {   // the imaging pass: ion_peel_direct at emission (ionizing_field_mod.f90:126, 157)
            auto kap_p = [&](int q) -> R {
                Col<R, NABS> cq;
                cq.load(a.col, q);
                R k = cq.template kappa<X>(s0, s1, s2, s3);
                if constexpr (METAL) {
                    if (a.metal_abs) k = k + mp.kappa(a.m, q, msg);
                }
                return k;
            };
            peel_direct<false>(a, rec.p0[i], rec.p0[c + i], rec.p0[2 * c + i], -1, inu, a.Lpacket, kap_p, bits);
        }
        // ring of LA+1 cells: il, segment, columns, and whether a next cell exists
        int il[LA + 1] = {};
        double sgm[LA + 1] = {};
        Col<R, NABS> cl[LA + 1];
        bool more[LA + 1];
        more[0] = g.emit(nx, ny, nz, &il[0], &sgm[0]);
        cl[0].load(a.col, il[0]);
#pragma unroll
        for (int k = 1; k <= LA; ++k) {
            more[k] = false;
            if (more[k - 1]) {
                more[k] = g.emit(nx, ny, nz, &il[k], &sgm[k]);
                cl[k].load(a.col, il[k]);
            }
        }
        R expo = (R)1.0;
        double tau = 0.0;
        int nstep = 0;
        bool out = false;   // left the grid through a face (not the tau or step limits)
        for (;;) {
            if (++nstep > kMaxWalkSteps) { ++kills; break; }
            R kap = cl[0].template kappa<X>(s0, s1, s2, s3);
            if constexpr (METAL) {
                if (a.metal_abs) kap = kap + mp.kappa(a.m, il[0], msg);
            }
            const R ks = kap * (R)sgm[0];
            R w;
            if (ks > (R)0) {
                w = segment_weight(expo, ks, kap);
            } else {
                w = expo * (R)sgm[0];
            }
            if (w != (R)0) {   // score_ion_path returns on a zero path (ion_score_mod.f90:148)
                ++nseg;
                nact += mp.nm;
                score_hhe<T, R, NT>(tal, jt, il[0], a.nnu, inu, w, cf);
                if constexpr (METAL) mp.template score<T>(a.m, il[0], w, msg, mhc);
            }
            tau = tau + (double)ks;
            if (tau >= kTauHuge) break;
            if constexpr (!X && sizeof(R) == 4) {
                if (expo == (R)0) break;   // FP32 attenuation underflowed: every later segment scores zero
            }
            if (!more[0]) { out = true; break; }   // the scored cell was the last one inside the grid
#pragma unroll
            for (int k = 0; k < LA; ++k) {
                il[k] = il[k + 1]; sgm[k] = sgm[k + 1]; cl[k] = cl[k + 1]; more[k] = more[k + 1];
            }
            if (LA == 0 || more[LA - (LA > 0)]) {
                more[LA] = g.emit(nx, ny, nz, &il[LA], &sgm[LA]);
                cl[LA].load(a.col, il[LA]);
            } else {
                more[LA] = false;
            }
        }
        // a z-face escape carries the surviving luminosity to the slab's
        // boundary tally (raytrace_amr.f90:586-588)
        if (out && a.slab_iesc) slab_add(a, rec.p0[5 * c + i], (double)expo * a.Lpacket);
        // ion_score_energy_packet (ion_score_mod.f90:233-252)
        const double lum = a.Lpacket;
        const double tr = exp(-fmax(tau, 0.0));
        emitted += lum;
        absorbed += lum * (1.0 - tr);
        escaped += lum * tr;
        if constexpr (X) {
            if (a.scatter && tau > 1.0e-12) {
                auto kappa_at = [&](int q) -> R {
                    Col<R, NABS> cq;
                    cq.load(a.col, q);
                    R k = cq.template kappa<X>(s0, s1, s2, s3);
                    if constexpr (METAL) {
                        if (a.metal_abs) k = k + mp.kappa(a.m, q, msg);
                    }
                    return k;
                };
                auto score_at = [&](int q, double pl) {
                    const R w = (R)pl;
                    if (w != (R)0) {
                        ++nscat;
                        nact += mp.nm;
                        score_hhe<T, R, NT>(tal, jt, q, a.nnu, inu, w, cf);
                        if constexpr (METAL) mp.template score<T>(a.m, q, w, msg, mhc);
                    }
                };
                const R* ds = static_cast<const R*>(rec.dsc);
                auto peel_at = [&](double px, double py, double pz, int q, double qx, double qy, double qz, double w) {
                    if (a.peeling)
                        peel_scatter<false>(a, px, py, pz, q, qx, qy, qz, a.Lpacket * w, (double)ds[c + i], inu, kappa_at);
                };
                scattered_flights<false>(a, rec.p0[i], rec.p0[c + i], rec.p0[2 * c + i], rec.p0[3 * c + i], rec.p0[4 * c + i],
                                         rec.p0[5 * c + i], -1, tau, (double)ds[i], (double)ds[c + i], (uint32_t)stream,
                                         (uint64_t)(ip0 + i), kappa_at, score_at, peel_at, kills);
            }
        }
    }
    walk_epilogue<METAL>(a, emitted, absorbed, escaped, nseg, kills, nact, nscat, accumulate, sh);
}

// ---- coherent walk with warp-aggregated tallies ----------------------------------
// Sum of v over the lanes of `peers` (the lanes holding this lane's key),
// left in the group's lowest lane, which the return value marks.  A pairwise
// tree over each group's lanes in lane order: every round each remaining lane
// adds the value of its next remaining peer, and the lanes whose rank in the
// group is odd drop out; ceil(log2(group size)) rounds, none when every lane
// is alone.  All 32 lanes must call it together.
template <typename A, int N>
__device__ __forceinline__ bool peer_sum(unsigned peers, int lane, A (&v)[N]) {
    const unsigned below = (1u << lane) - 1u;
    unsigned rest = peers & ~(below | (1u << lane));   // peers above this lane
    int rank = __popc(peers & below);
    while (__any_sync(0xffffffffu, rest != 0u)) {
        const int next = __ffs(rest);                  // 1 + lane of the next remaining peer, 0: none
        const int src = next ? next - 1 : lane;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const A t = __shfl_sync(0xffffffffu, v[k], src);
            if (next) v[k] += t;
        }
        const bool done = rank & 1;
        const unsigned keep = __ballot_sync(0xffffffffu, !done);
        rest = done ? 0u : (rest & keep);
        rank >>= 1;
    }
    return (peers & below) == 0u;
}

// Walk kernel of packet_order 'coherent' (raytrace_ion_to_edge_car,
// raytrace_amr.f90:534-592, and score_ion_path, ion_score_mod.f90:137-231):
// each warp walks 32 consecutive packets of the sorted chunk -- nearly
// parallel rays of nearly equal energy -- in step with one another.  Every
// step the lanes that score the same (leaf, spectrum bin, moment bin) are
// found with one match and their path luminosities summed over the warp, so
// each distinct tally sector takes one reduction instead of one per lane:
// the H/He rate tallies, the spectrum bin and (MET 2) the six energy
// moments.  Exact metal tallies (MET 1) stay per lane.  The leaf sequences,
// segments and energy ledger are those of k_walk_edge; only the summation
// order of the tallies differs.  No grain or FUV terms (X = 0).
template <typename R, int NABS, int LA, int MET, typename T>
__global__ void __launch_bounds__(128) k_walk_coh(const PassArgs a, const PacketRecords rec, long long n,
                                                  int accumulate) {
    constexpr int NT = NABS == 1 ? 2 : 6;
    constexpr bool METAL = MET > 0;
    constexpr int NM = MET == 2 ? kMomDeg : 0;      // moment values aggregated per step
    constexpr int NV = NT + 1 + NM;                  // + the spectrum bin
    __shared__ double sh[128];
    extern __shared__ __align__(16) unsigned char dsm[];
    R* const msg = reinterpret_cast<R*>(dsm);
    R* const mhc = msg + (MET == 1 ? a.m.ntrp * blockDim.x : 0);
    double emitted = 0.0, absorbed = 0.0, escaped = 0.0;
    unsigned long long nseg = 0, kills = 0, nact = 0, nscat = 0;
    T* tal = static_cast<T*>(a.tally);
    T* jt = static_cast<T*>(a.jt);
    const R* sg = static_cast<const R*>(rec.sig);
    const R* cfp = static_cast<const R*>(rec.coef);
    const long long c = rec.cap;
    const int nx = a.n[0], ny = a.n[1], nz = a.n[2];
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const unsigned long long nnu = (unsigned long long)a.nnu;
    const unsigned long long nmb = MET == 2 ? (unsigned long long)a.m.nmb : 1ull;
    for (long long base = warp * 32; base < n; base += nwarps * 32) {
        const long long i = base + lane;
        bool alive = i < n;
        const long long ir = alive ? i : base;   // a lane past the chunk end reads a valid record and idles
        Stepper g;
        g.t0 = rec.tm[ir]; g.t1 = rec.tm[c + ir]; g.t2 = rec.tm[2 * c + ir];
        g.d0 = rec.td[ir]; g.d1 = rec.td[c + ir]; g.d2 = rec.td[2 * c + ir];
        g.t_cur = 0.0;
        g.per = a.xyper;
        const int cell = rec.cell[ir], bits = rec.bits[ir];
        g.ix = cell & 1023; g.iy = (cell >> 10) & 1023; g.iz = (cell >> 20) & 1023;
        g.sx = ((bits >> 16) & 3) - 1; g.sy = ((bits >> 18) & 3) - 1; g.sz = ((bits >> 20) & 3) - 1;
        const int inu = bits & 0xFFFF;
        const R s0 = sg[ir];
        const R s1 = NABS == 1 ? (R)0 : sg[c + ir];
        const R s2 = NABS == 1 ? (R)0 : sg[2 * c + ir];
        R cf[NT];
#pragma unroll
        for (int k = 0; k < NT; ++k) cf[k] = cfp[k * c + ir];
        MetalPacket<R, MET> mp;
        if constexpr (METAL) mp.setup(a.m, rec, ir, msg, mhc);
        int il[LA + 1] = {};
        double sgm[LA + 1] = {};
        Col<R, NABS> cl[LA + 1];
        bool more[LA + 1];
        more[0] = g.emit(nx, ny, nz, &il[0], &sgm[0]);
        cl[0].load(a.col, il[0]);
#pragma unroll
        for (int k = 1; k <= LA; ++k) {
            more[k] = false;
            if (more[k - 1]) {
                more[k] = g.emit(nx, ny, nz, &il[k], &sgm[k]);
                cl[k].load(a.col, il[k]);
            }
        }
        R expo = (R)1.0;
        double tau = 0.0;
        int nstep = 0;
        while (__any_sync(0xffffffffu, alive)) {
            R w = (R)0;
            bool finish = false;
            if (alive) {
                if (++nstep > kMaxWalkSteps) {
                    ++kills;
                    finish = true;
                } else {
                    R kap = cl[0].template kappa<0>(s0, s1, s2, (R)0);
                    if constexpr (METAL) {
                        if (a.metal_abs) kap = kap + mp.kappa(a.m, il[0], msg);
                    }
                    const R ks = kap * (R)sgm[0];
                    if (ks > (R)0) {
                        w = segment_weight(expo, ks, kap);
                    } else {
                        w = expo * (R)sgm[0];
                    }
                    tau = tau + (double)ks;
                    // an FP32 attenuation that underflowed scores zero on every later segment
                    finish = tau >= kTauHuge || !more[0] || (sizeof(R) == 4 && expo == (R)0);
                }
            }
            // score_ion_path over the warp: one reduction per distinct key
            const bool scored = w != (R)0;   // score_ion_path returns on a zero path (ion_score_mod.f90:148)
            const unsigned long long key =
                scored ? (((unsigned long long)il[0] * nmb + (unsigned long long)mp.mb) * nnu + (unsigned long long)inu)
                       : ~(unsigned long long)lane;
            const unsigned peers = __match_any_sync(0xffffffffu, key);
            R v[NV];
#pragma unroll
            for (int k = 0; k < NT; ++k) v[k] = w * cf[k];
            v[NT] = w;
            if constexpr (MET == 2) {
#pragma unroll
                for (int q = 0; q < NM; ++q) v[NT + 1 + q] = w * mp.phi[q];
            }
            const bool lead = peer_sum<R, NV>(peers, lane, v);
            if (scored) {
                ++nseg;
                nact += mp.nm;
                if (lead) {
                    T* tl = tal + (long long)il[0] * NT;
#pragma unroll
                    for (int k = 0; k < NT; ++k) tally_add(tl + k, v[k]);
                    tally_add(jt + (long long)il[0] * a.nnu + inu, v[NT]);
                    if constexpr (MET == 2) {
                        bool vec = false;
                        if constexpr (std::is_same<R, float>::value && std::is_same<T, double>::value) {
                            if (a.m.mom32) {   // FP32 moments: one sector, two vector reductions
                                float* mt = static_cast<float*>(a.m.mom) + ((long long)il[0] * a.m.nmb + mp.mb) * 8;
                                asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(mt),
                                             "f"(v[NT + 1]), "f"(v[NT + 2]), "f"(v[NT + 3]), "f"(v[NT + 4])
                                             : "memory");
                                asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(mt + 4), "f"(v[NT + 5]),
                                             "f"(v[NT + 6])
                                             : "memory");
                                vec = true;
                            }
                        }
                        if (!vec) {
                            T* mt = static_cast<T*>(a.m.mom) + ((long long)il[0] * a.m.nmb + mp.mb) * kMomDeg;
#pragma unroll
                            for (int q = 0; q < kMomDeg; ++q) tally_add(mt + q, v[NT + 1 + q]);
                        }
                    }
                }
                if constexpr (MET == 1) mp.template score<T>(a.m, il[0], w, msg, mhc);
            }
            if (alive) {
                if (finish) {   // ion_score_energy_packet (ion_score_mod.f90:233-252)
                    const double lum = a.Lpacket;
                    const double tr = exp(-fmax(tau, 0.0));
                    emitted += lum;
                    absorbed += lum * (1.0 - tr);
                    escaped += lum * tr;
                    alive = false;
                } else {
#pragma unroll
                    for (int k = 0; k < LA; ++k) {
                        il[k] = il[k + 1]; sgm[k] = sgm[k + 1]; cl[k] = cl[k + 1]; more[k] = more[k + 1];
                    }
                    if (LA == 0 || more[LA - (LA > 0)]) {
                        more[LA] = g.emit(nx, ny, nz, &il[LA], &sgm[LA]);
                        cl[LA].load(a.col, il[LA]);
                    } else {
                        more[LA] = false;
                    }
                }
            }
        }
    }
    walk_epilogue<METAL>(a, emitted, absorbed, escaped, nseg, kills, nact, nscat, accumulate, sh);
}

// Walk kernel on the octree: raytrace_ion_to_edge_amr (raytrace_amr.f90:
// 422-486, without the xy-periodic wrap) for the packets of one chunk,
// grid-stride.  Per segment: the leaf's geometry record and columns (both
// leaf-indexed, issued together), the exit face (amr_cell_exit), the
// attenuated path score, the move to the exit point, and the leaf across the
// face (amr_next_leaf).  Geometry in FP64 without contraction, as the
// reference's.  MET, X, ip0 and stream as for k_walk_edge.
template <typename R, int NABS, int MET, int X, typename T>
__global__ void __launch_bounds__(128) k_walk_amr(const PassArgs a, const PacketRecords rec, long long n,
                                                  int accumulate, long long ip0, int stream) {
    constexpr int NT = X ? 8 : (NABS == 1 ? 2 : 6);
    constexpr bool METAL = MET > 0;
    __shared__ double sh[128];
    extern __shared__ __align__(16) unsigned char dsm[];
    R* const msg = reinterpret_cast<R*>(dsm);
    R* const mhc = msg + (MET == 1 ? a.m.ntrp * blockDim.x : 0);
    double emitted = 0.0, absorbed = 0.0, escaped = 0.0;
    unsigned long long nseg = 0, kills = 0, nact = 0, nscat = 0;
    T* tal = static_cast<T*>(a.tally);
    T* jt = static_cast<T*>(a.jt);
    const R* sg = static_cast<const R*>(rec.sig);
    const R* cfp = static_cast<const R*>(rec.coef);
    const long long c = rec.cap;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const long long i = rec.perm ? (long long)rec.perm[j] : j;
        double x = rec.tm[i], y = rec.tm[c + i], z = rec.tm[2 * c + i];
        const double kx = rec.td[i], ky = rec.td[c + i], kz = rec.td[2 * c + i];
        int il = rec.cell[i];
        const int inu = rec.bits[i] & 0xFFFF;
        const R s0 = sg[i];
        const R s1 = NABS == 1 ? (R)0 : sg[c + i];
        const R s2 = NABS == 1 ? (R)0 : sg[2 * c + i];
        const R s3 = X ? sg[3 * c + i] : (R)0;
        R cf[NT];
#pragma unroll
        for (int k = 0; k < NT; ++k) cf[k] = cfp[k * c + i];
        MetalPacket<R, MET> mp;
        if constexpr (METAL) mp.setup(a.m, rec, i, msg, mhc);
        if (a.peeling) {   // the imaging pass: ion_peel_direct at emission (ionizing_field_mod.f90:126, 157)
            auto kap_p = [&](int q) -> R {
                Col<R, NABS> cq;
                cq.load(a.col, q);
                R k = cq.template kappa<X>(s0, s1, s2, s3);
                if constexpr (METAL) {
                    if (a.metal_abs) k = k + mp.kappa(a.m, q, msg);
                }
                return k;
            };
            peel_direct<true>(a, x, y, z, il, inu, a.Lpacket, kap_p, rec.bits[i]);
        }
        R expo = (R)1.0;
        double tau = 0.0;
        int nstep = 0;
        int face = -1;   // the face the last leaf was left by; il < 0 after it: out of the grid
        while (il >= 0) {
            if (++nstep > kMaxWalkSteps) { ++kills; break; }
            const double4 g = ld_geo(a.oct.lgeo + il);
            Col<R, NABS> cl;
            cl.load(a.col, il);
            const double texit = oct_cell_exit(g, x, y, z, kx, ky, kz, &face);
            R kap = cl.template kappa<X>(s0, s1, s2, s3);
            if constexpr (METAL) {
                if (a.metal_abs) kap = kap + mp.kappa(a.m, il, msg);
            }
            const R ks = kap * (R)texit;
            R w;
            if (ks > (R)0) {
                w = segment_weight(expo, ks, kap);
            } else {
                w = expo * (R)texit;
            }
            if (w != (R)0) {
                ++nseg;
                nact += mp.nm;
                score_hhe<T, R, NT>(tal, jt, il, a.nnu, inu, w, cf);
                if constexpr (METAL) mp.template score<T>(a.m, il, w, msg, mhc);
            }
            tau = tau + (double)ks;
            if (tau >= kTauHuge) break;
            if constexpr (!X && sizeof(R) == 4) {
                if (expo == (R)0) break;   // FP32 attenuation underflowed: every later segment scores zero
            }
            x = x + texit * kx;
            y = y + texit * ky;
            z = z + texit * kz;
            il = oct_next_leaf(a.oct, il, face, x, y, z);
            if (il < 0 && a.xyper) {   // raytrace_amr.f90:473-476
                slab_wrap_xy(a, face, x, y);
                if (face <= 3) il = oct_find_leaf(a.oct, x, y, z);
            }
        }
        // a z-face escape carries the surviving luminosity to the slab's
        // boundary tally (raytrace_amr.f90:477-481)
        if (il < 0 && face >= 4 && a.slab_iesc) slab_add(a, kz, (double)expo * a.Lpacket);
        const double lum = a.Lpacket;
        const double tr = exp(-fmax(tau, 0.0));
        emitted += lum;
        absorbed += lum * (1.0 - tr);
        escaped += lum * tr;
        if constexpr (X) {
            if (a.scatter && tau > 1.0e-12) {
                auto kappa_at = [&](int q) -> R {
                    Col<R, NABS> cq;
                    cq.load(a.col, q);
                    R k = cq.template kappa<X>(s0, s1, s2, s3);
                    if constexpr (METAL) {
                        if (a.metal_abs) k = k + mp.kappa(a.m, q, msg);
                    }
                    return k;
                };
                auto score_at = [&](int q, double pl) {
                    const R w = (R)pl;
                    if (w != (R)0) {
                        ++nscat;
                        nact += mp.nm;
                        score_hhe<T, R, NT>(tal, jt, q, a.nnu, inu, w, cf);
                        if constexpr (METAL) mp.template score<T>(a.m, q, w, msg, mhc);
                    }
                };
                const R* ds = static_cast<const R*>(rec.dsc);
                auto peel_at = [&](double px, double py, double pz, int q, double qx, double qy, double qz, double w) {
                    if (a.peeling)
                        peel_scatter<true>(a, px, py, pz, q, qx, qy, qz, a.Lpacket * w, (double)ds[c + i], inu, kappa_at);
                };
                scattered_flights<true>(a, rec.tm[i], rec.tm[c + i], rec.tm[2 * c + i], kx, ky, kz, rec.cell[i], tau,
                                        (double)ds[i], (double)ds[c + i], (uint32_t)stream, (uint64_t)(ip0 + i),
                                        kappa_at, score_at, peel_at, kills);
            }
        }
    }
    walk_epilogue<METAL>(a, emitted, absorbed, escaped, nseg, kills, nact, nscat, accumulate, sh);
}

// gas_rates_compute + ion_score_apply_hhe (gas_rates_mod.f90:82-153,
// ion_score_mod.f90:298-317): Gamma = sum * Lpacket * 1e-18 / ev2erg * fac,
// H = sum * Lpacket * 1e-18 * fac, fac = 1/((2h)^3 distance2cm^2).  The
// FP32 pair is reduced in FP64 here.
template <typename T>
__device__ __forceinline__ double tval(const T& v);
template <> __device__ __forceinline__ double tval<double>(const double& v) { return v; }
template <> __device__ __forceinline__ double tval<float>(const float& v) { return (double)v; }
template <> __device__ __forceinline__ double tval<float2>(const float2& v) { return (double)v.x + (double)v.y; }

//
// On the octree the leaf volume varies: cg, ch exclude fac and each leaf
// multiplies by its own 1/((2h)^3 d2), lg = the leaf geometry records.
__device__ __forceinline__ double leaf_fac(const double4* lg, long long il, double d2) {
    if (!lg) return 1.0;
    const double w = 2.0 * ld_geo(lg + il).w;
    return 1.0 / ((w * w * w) * d2);
}

//
// NT = 8 adds ion_score_apply_dust_heat and ion_score_apply_g0
// (ion_score_mod.f90:319-355): heat_dust = sum(w s_abs) Lpacket fac rhokap /
// distance2cm and G0 = sum_FUV(w) Lpacket fac / 1.6e-3, rows 6 and 7.
template <typename T, int NT>
__global__ void k_rates(const T* __restrict__ tal, double* __restrict__ rates, long long nleaf, double cg0, double ch0,
                        const double4* lg, double d2, const double* __restrict__ rhokap, double d2cm) {
    for (long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x; il < nleaf;
         il += (long long)gridDim.x * blockDim.x) {
        const double f = leaf_fac(lg, il, d2);
        const double cg = cg0 * f, ch = ch0 * f;
        const T* t = tal + il * NT;
        rates[0 * nleaf + il] = tval<T>(t[0]) * cg;
        rates[3 * nleaf + il] = tval<T>(t[1]) * ch;
        if (NT >= 6) {
            rates[1 * nleaf + il] = tval<T>(t[2]) * cg;
            rates[4 * nleaf + il] = tval<T>(t[3]) * ch;
            rates[2 * nleaf + il] = tval<T>(t[4]) * cg;
            rates[5 * nleaf + il] = tval<T>(t[5]) * ch;
            if (NT == 8) {
                const double lf = ch * 1.0e18;   // Lpacket x fac
                rates[6 * nleaf + il] = rhokap ? tval<T>(t[6]) * lf * rhokap[il] / d2cm : 0.0;
                rates[7 * nleaf + il] = tval<T>(t[7]) * lf / 1.6e-3;
            }
        } else {
            rates[1 * nleaf + il] = 0.0;
            rates[4 * nleaf + il] = 0.0;
            rates[2 * nleaf + il] = 0.0;
            rates[5 * nleaf + il] = 0.0;
        }
    }
}

template <typename T>
__global__ void k_jt(const T* __restrict__ jt, double* __restrict__ out, long long n, double scale) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = tval<T>(jt[i]) * scale;
}

// species_gamma_compute (species_mod.f90:493-512): per-leaf metal Gamma and
// photoheating from the path tallies, into element order.
template <typename T>
__global__ void k_metal_rates(const MetalDev m, long long nleaf, double cg, double ch, const double4* lg, double d2) {
    const T* raw = static_cast<const T*>(m.raw);
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nleaf * m.ntr;
         q += (long long)gridDim.x * blockDim.x) {
        const long long il = q / m.ntr;
        const int j = (int)(q - il * m.ntr);
        const int k = m.tr[j].flat;
        const T* r = raw + (il * m.ntrp + k) * 2;
        const double f = leaf_fac(lg, il, d2);
        m.egam[q] = tval<T>(r[0]) * (cg * f);
        m.eheat[q] = tval<T>(r[1]) * (ch * f);
    }
}

// The same from the energy moments: raw_{k,c}(leaf) = sum over the moment
// bins b and Chebyshev orders q of mom(leaf, b, q) * coef(b, q, k, c), as a
// tiled product of the (leaves x nmb*kMomDeg) moments with the
// (nmb*kMomDeg x 2 ntrp) coefficients.  A transition's coefficients are zero
// below its first active bin, so the dense sum adds the bin-restricted sum's
// terms in the same order (b, then q, ascending) and zeros before them.
// Block: 64 leaves x all outputs, 256 threads, each 4 leaves x NU outputs;
// the moments and coefficients staged through shared memory KC orders at a
// time.  RS: the words per (leaf, bin) in the tally (kMomDeg, or 8 for the
// padded FP32 moments).
constexpr int kRtM = 64, kRtThreads = 256;

template <typename T, int NU, int KC, int RS>
__global__ void __launch_bounds__(kRtThreads) k_metal_rates_mom(const MetalDev m, long long nleaf, double cg,
                                                                double ch, const double4* lg, double d2) {
    __shared__ double sA[kRtM][KC + 1];
    __shared__ double sB[KC][16 * NU];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int K = m.nmb * kMomDeg, N = 2 * m.ntrp;
    const T* mom = static_cast<const T*>(m.mom);
    const double* C = m.mcoef;   // [K][ntrp][2] = K x N, row-major
    for (long long tile = blockIdx.x; tile * kRtM < nleaf; tile += gridDim.x) {
        const long long l0 = tile * kRtM;
        double acc[4][NU];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int u = 0; u < NU; ++u) acc[i][u] = 0.0;
        for (int k0 = 0; k0 < K; k0 += KC) {
            __syncthreads();
            for (int e = tid; e < kRtM * KC; e += kRtThreads) {
                const int r = e / KC, q = e - r * KC;
                const long long il = l0 + r;
                const int kk = k0 + q;
                const int bin = kk / kMomDeg;
                sA[r][q] = (il < nleaf && kk < K)
                               ? tval<T>(mom[il * ((long long)m.nmb * RS) + bin * RS + (kk - bin * kMomDeg)])
                               : 0.0;
            }
            for (int e = tid; e < KC * 16 * NU; e += kRtThreads) {
                const int r = e / (16 * NU), q = e - r * (16 * NU);
                const int kk = k0 + r;
                sB[r][q] = (kk < K && q < N) ? __ldg(C + (size_t)kk * N + q) : 0.0;
            }
            __syncthreads();
            const int kn = min(KC, K - k0);
            for (int kk = 0; kk < kn; ++kk) {
                double a[4], b[NU];
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] = sA[ty * 4 + i][kk];
#pragma unroll
                for (int u = 0; u < NU; ++u) b[u] = sB[kk][tx + 16 * u];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int u = 0; u < NU; ++u) acc[i][u] = acc[i][u] + a[i] * b[u];
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const long long il = l0 + ty * 4 + i;
            if (il >= nleaf) continue;
            const double f = leaf_fac(lg, il, d2);
#pragma unroll
            for (int u = 0; u < NU; ++u) {
                const int col = tx + 16 * u;
                if (col >= N) continue;
                const int j = m.jof[col >> 1];
                if (j < 0) continue;
                if (col & 1) m.eheat[il * m.ntr + j] = acc[i][u] * (ch * f);
                else m.egam[il * m.ntr + j] = acc[i][u] * (cg * f);
            }
        }
    }
}

// Sobol uniforms for the test hook.
__global__ void k_sobol(const QmcTables* t, int stream, long long idx0, long long n, int nd, double* out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        for (int d = 0; d < nd; ++d) out[i * nd + d] = qmc_uniform(*t, (uint64_t)(idx0 + i), d, stream);
}

// Draws n0 .. n0+n-1 of one packet's Philox stream, for the test hook (one
// thread walks the stream in order, as a packet does).
__global__ void k_philox(unsigned long long seed, unsigned stream, unsigned long long packet, int n0, int n,
                         double* out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    PacketStream rs;
    rs.init(seed, stream, packet);
    for (int k = 0; k < n0 + n; ++k) {
        const double u = rs.next();
        if (k >= n0) out[k - n0] = u;
    }
}

// Geometry-only DDA (no optical-depth cut) for the leaf-sequence hook.
__global__ void k_walk(const double* rays, long long nray, int max_steps, int* leaves, int* nsteps, double ox,
                       double oy, double oz, double d, int nx, int ny, int nz) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nray) return;
    const double pos[3] = {rays[6 * r], rays[6 * r + 1], rays[6 * r + 2]};
    const double kk[3] = {rays[6 * r + 3], rays[6 * r + 4], rays[6 * r + 5]};
    const double org[3] = {ox, oy, oz};
    const int n[3] = {nx, ny, nz};
    int idx[3], stp[3];
    double tmax[3], tdel[3];
    for (int k = 0; k < 3; ++k) {
        idx[k] = min(max((int)((pos[k] - org[k]) / d), 0), n[k] - 1);
        if (kk[k] > 0.0) {
            stp[k] = 1; tmax[k] = (org[k] + (double)(idx[k] + 1) * d - pos[k]) / kk[k]; tdel[k] = d / kk[k];
        } else if (kk[k] < 0.0) {
            stp[k] = -1; tmax[k] = (org[k] + (double)idx[k] * d - pos[k]) / kk[k]; tdel[k] = -d / kk[k];
        } else {
            stp[k] = 0; tmax[k] = kHugest; tdel[k] = kHugest;
        }
    }
    int ns = 0;
    while (ns < max_steps) {
        leaves[r * max_steps + ns++] = idx[0] + n[0] * (idx[1] + n[1] * idx[2]);
        int ax = 0;
        if (tmax[1] < tmax[ax]) ax = 1;
        if (tmax[2] < tmax[ax]) ax = 2;
        tmax[ax] = tmax[ax] + tdel[ax];
        idx[ax] += stp[ax];
        if (idx[ax] < 0 || idx[ax] >= n[ax]) break;
    }
    nsteps[r] = ns;
    for (int s = ns; s < max_steps; ++s) leaves[r * max_steps + s] = -1;
}

// Geometry-only octree walk for the leaf-sequence hook: amr_find_leaf at the
// start point, then amr_cell_exit / amr_next_leaf to the box edge.
__global__ void k_walk_amr_leaves(const double* rays, long long nray, int max_steps, int* leaves, int* nsteps,
                                  const OctDev o) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nray) return;
    double x = rays[6 * r], y = rays[6 * r + 1], z = rays[6 * r + 2];
    const double kx = rays[6 * r + 3], ky = rays[6 * r + 4], kz = rays[6 * r + 5];
    int il = oct_find_leaf(o, x, y, z), ns = 0;
    while (il >= 0 && ns < max_steps) {
        leaves[r * max_steps + ns++] = il;
        int face;
        const double t = oct_cell_exit(ld_geo(o.lgeo + il), x, y, z, kx, ky, kz, &face);
        x = x + t * kx;
        y = y + t * ky;
        z = z + t * kz;
        il = oct_next_leaf(o, il, face, x, y, z);
    }
    nsteps[r] = ns;
    for (int s = ns; s < max_steps; ++s) leaves[r * max_steps + s] = -1;
}

// Launch records (x, y, z, kx, ky, kz, E, inu) for the launch hook.
__global__ void k_launch_records(const PassArgs a, long long ip0, long long n, double* out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long ip = ip0 + i;
    double u[7];
    for (int d = 0; d < a.ndim; ++d) u[d] = qmc_uniform(*a.qmc, (uint64_t)ip, d, 0);
    int ic;
    double E, pos[3], kk[3];
    launch_packet(a, u, ic, E, pos, kk);
    double* o = out + 8 * i;
    o[0] = pos[0]; o[1] = pos[1]; o[2] = pos[2];
    o[3] = kk[0]; o[4] = kk[1]; o[5] = kk[2];
    o[6] = E;
    o[7] = (double)bin_of(a.eedge, a.nnu, E);
}

PassArgs make_args(mochii_ctx* c) {
    PassArgs a;
    a.qmc = c->tab.qmc;
    a.tab_e = c->tab.tab_e;
    a.tab_f = c->tab.tab_f;
    a.tab_c = c->tab.tab_c;
    a.tab_off = c->tab.tab_off;
    a.comp = c->tab.comp;
    a.eedge = c->tab.eedge;
    a.col = c->col;
    a.tally = c->tally;
    a.jt = c->jt;
    a.ledger = c->tw.ledger;
    a.counters = c->tw.counters;
    a.np = c->par.nphotons;
    a.Lpacket = c->band.ion_Ltot / (double)c->par.nphotons;
    a.org[0] = c->grid.xmin; a.org[1] = c->grid.ymin; a.org[2] = c->grid.zmin;
    a.dcell = c->grid.dcell;
    a.n[0] = c->grid.nx; a.n[1] = c->grid.ny; a.n[2] = c->grid.nz;
    a.ncomp = c->band.ncomp;
    a.multi = c->band.multi;
    a.ndim = c->band.qmc_ndim;
    a.ext_ic = c->band.ext_ic;
    a.ext_sph = c->band.ext_sph;
    a.ext_rmax = c->par.rmax;
    a.bmin[0] = c->grid.xmin; a.bmin[1] = c->grid.ymin; a.bmin[2] = c->grid.zmin;
    a.bmax[0] = c->grid.xmax; a.bmax[1] = c->grid.ymax; a.bmax[2] = c->grid.zmax;
    a.xyper = c->par.xy_periodic ? 1 : 0;
    a.slab = c->band.slab;
    for (int f = 0; f < 2; ++f) {
        a.slab_mode[f] = c->band.slab_mode[f];
        a.slab_mu[f] = c->band.slab_mu[f];
        a.slab_phi[f] = c->band.slab_phi[f];
    }
    a.slab_ptop = c->band.slab_ptop;
    a.slab_nmu = c->band.slab ? c->par.slab_nmu : 0;
    a.slab_iesc = c->band.slab ? c->slab_iesc : nullptr;
    a.nnu = c->nnu;
    a.m = c->metal;
    a.metal_abs = c->par.ion_metal_abs;
    a.oct = c->oct;
    a.dust = c->dust;
    a.rhokap = c->rhokap;
    a.xs = c->xscore ? 1 : 0;
    a.scatter = c->scatter ? 1 : 0;
    a.eion_min = c->par.eion_min;
    a.seed = (unsigned long long)(long long)c->par.random_seed;
    a.peel = c->peel;
    a.peeling = c->peeling ? 1 : 0;
    return a;
}

int grid_blocks(long long work, int threads, int cap) {
    long long b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

}  // namespace

// Dynamic shared memory of the metal walk: sigma_k (and sigma_k h_k for the
// exact tallies) per thread.
size_t metal_smem(const mochii_ctx* c) {
    if (c->metal.ntr == 0) return 0;
    return (c->metal.nmb > 0 ? 1 : 2) * (size_t)c->metal.ntrp * 128 * (c->fp32 ? 4 : 8);
}

// Absorber variants of the walk kernels: V = 1 (H I), 4 (H I, He I, He II),
// 5 (4 + grains and FUV: X).
template <int V> struct AbsV {
    static constexpr int NABS = V == 1 ? 1 : 4;
    static constexpr int X = V == 5 ? 1 : 0;
};

int abs_variant(const mochii_ctx* c) { return c->xscore ? 5 : c->nabs == 1 ? 1 : 4; }

template <typename R, typename T, int V, int LA, int MET>
int walk_occupancy(size_t smem) {
    auto k = k_walk_edge<R, AbsV<V>::NABS, LA, MET, AbsV<V>::X, T>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, 128, smem) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return nb > 0 ? nb : 1;
}

template <typename R, typename T>
int walk_occupancy_any(const mochii_ctx* c, size_t smem) {
    switch (abs_variant(c)) {
        case 1: return walk_occupancy<R, T, 1, 2, 1>(smem);
        case 4: return walk_occupancy<R, T, 4, 2, 1>(smem);
        default: return walk_occupancy<R, T, 5, 2, 1>(smem);
    }
}

int transport_blocks(const mochii_ctx* c) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    int per_sm = c->tune.walk_blocks_per_sm > 0 ? c->tune.walk_blocks_per_sm : 8;
    if (c->metal.ntr > 0) {   // resident blocks only: each holds its packets' sigma_k in shared memory
        const size_t smem = metal_smem(c);
        const int occ = !c->fp32 ? walk_occupancy_any<double, double>(c, smem)
                        : c->tally64 ? walk_occupancy_any<float, double>(c, smem)
                                     : walk_occupancy_any<float, float2>(c, smem);
        per_sm = per_sm < occ ? per_sm : occ;
    }
    return grid_blocks(c->par.nphotons, 128, sms * per_sm);
}

// One chunk's walk: packets ip0 .. ip0 + n - 1 of a stream (0 stellar, 1
// diffuse), accumulate into the per-block ledger unless acc == 0.
struct WalkLaunch {
    long long n, ip0;
    int acc, blocks, stream;
    bool coherent = false;   // records in coherent_key order, walked by k_walk_coh
};

// packet_order 'coherent' applies to the stellar and the diffuse packets on
// the Cartesian grid without grain or FUV terms; elsewhere the launch order
// is walked.
bool coherent_walk_applies(const mochii_ctx* c) {
    return c->par.packet_order == 2 && c->oct.ncells == 0 && !c->xscore && c->rec.key != nullptr && !c->peeling &&
           !c->band.slab;
}

// Walk-kernel variants: look-ahead depth 0..2 (the autotuned choice is
// c->tune.lookahead); 128-thread blocks.
template <typename R, typename T, int V, int MET>
cudaError_t walk_la(mochii_ctx* c, const PassArgs& a, const PacketRecords& r, const WalkLaunch& w) {
    constexpr int NABS = AbsV<V>::NABS, X = AbsV<V>::X;
    const size_t smem = MET ? metal_smem(c) : 0;
    if (MET && smem > 48 * 1024) {
        cudaFuncSetAttribute(k_walk_edge<R, NABS, 0, MET, X, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_walk_edge<R, NABS, 1, MET, X, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_walk_edge<R, NABS, 2, MET, X, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    switch (c->tune.lookahead) {
        case 0: k_walk_edge<R, NABS, 0, MET, X, T><<<w.blocks, 128, smem, c->stream>>>(a, r, w.n, w.acc, w.ip0, w.stream); break;
        case 1: k_walk_edge<R, NABS, 1, MET, X, T><<<w.blocks, 128, smem, c->stream>>>(a, r, w.n, w.acc, w.ip0, w.stream); break;
        default: k_walk_edge<R, NABS, 2, MET, X, T><<<w.blocks, 128, smem, c->stream>>>(a, r, w.n, w.acc, w.ip0, w.stream); break;
    }
    return cudaGetLastError();
}

// The coherent walk (packet_order 'coherent', no grains): look-ahead 0..2.
template <typename R, typename T, int V, int MET>
cudaError_t walk_coh(mochii_ctx* c, const PassArgs& a, const PacketRecords& r, const WalkLaunch& w) {
    constexpr int NABS = AbsV<V>::NABS;
    const size_t smem = MET ? metal_smem(c) : 0;
    if (MET && smem > 48 * 1024) {
        cudaFuncSetAttribute(k_walk_coh<R, NABS, 0, MET, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_walk_coh<R, NABS, 1, MET, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(k_walk_coh<R, NABS, 2, MET, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    switch (c->tune.lookahead) {
        case 0: k_walk_coh<R, NABS, 0, MET, T><<<w.blocks, 128, smem, c->stream>>>(a, r, w.n, w.acc); break;
        case 1: k_walk_coh<R, NABS, 1, MET, T><<<w.blocks, 128, smem, c->stream>>>(a, r, w.n, w.acc); break;
        default: k_walk_coh<R, NABS, 2, MET, T><<<w.blocks, 128, smem, c->stream>>>(a, r, w.n, w.acc); break;
    }
    return cudaGetLastError();
}

// The octree walk: no look-ahead variants.
template <typename R, typename T, int V, int MET>
cudaError_t walk_amr(mochii_ctx* c, const PassArgs& a, const PacketRecords& r, const WalkLaunch& w) {
    constexpr int NABS = AbsV<V>::NABS, X = AbsV<V>::X;
    const size_t smem = MET ? metal_smem(c) : 0;
    if (MET && smem > 48 * 1024)
        cudaFuncSetAttribute(k_walk_amr<R, NABS, MET, X, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_walk_amr<R, NABS, MET, X, T><<<w.blocks, 128, smem, c->stream>>>(a, r, w.n, w.acc, w.ip0, w.stream);
    return cudaGetLastError();
}

template <typename R, typename T, int MET>
cudaError_t walk_abs(mochii_ctx* c, const PassArgs& a, const PacketRecords& r, const WalkLaunch& w) {
    const bool amr = c->oct.ncells > 0;
    if (w.coherent) {   // Cartesian grid, no grain or FUV terms (coherent_walk_applies)
        if (abs_variant(c) == 1) return walk_coh<R, T, 1, MET>(c, a, r, w);
        return walk_coh<R, T, 4, MET>(c, a, r, w);
    }
    switch (abs_variant(c)) {
        case 1: return amr ? walk_amr<R, T, 1, MET>(c, a, r, w) : walk_la<R, T, 1, MET>(c, a, r, w);
        case 4: return amr ? walk_amr<R, T, 4, MET>(c, a, r, w) : walk_la<R, T, 4, MET>(c, a, r, w);
        default: return amr ? walk_amr<R, T, 5, MET>(c, a, r, w) : walk_la<R, T, 5, MET>(c, a, r, w);
    }
}

template <typename R, typename T>
cudaError_t walk_prec(mochii_ctx* c, const PassArgs& a, const PacketRecords& r, const WalkLaunch& w) {
    if (c->metal.ntr == 0) return walk_abs<R, T, 0>(c, a, r, w);
    return c->metal.nmb > 0 ? walk_abs<R, T, 2>(c, a, r, w) : walk_abs<R, T, 1>(c, a, r, w);
}

// Segment arithmetic R and tally type T: FP64 / FP64; FP32 with FP64 tallies
// (tally64); FP32 with compensated FP32 pairs.
cudaError_t launch_walk_variant(mochii_ctx* c, const PassArgs& a, const PacketRecords& r, const WalkLaunch& w) {
    if (!c->fp32) return walk_prec<double, double>(c, a, r, w);
    return c->tally64 ? walk_prec<float, double>(c, a, r, w) : walk_prec<float, float2>(c, a, r, w);
}

PacketRecords packet_records(mochii_ctx* c) {
    PacketRecords r;
    r.cap = c->rec.cap;
    r.tm = c->rec.tm;
    r.td = c->rec.td;
    r.cell = c->rec.cell;
    r.bits = c->rec.bits;
    r.sig = c->rec.sig;
    r.coef = c->rec.coef;
    r.E = c->rec.E;
    r.msig = c->rec.msig;
    r.dsc = c->rec.dsc;
    r.p0 = c->rec.p0;
    r.key = c->par.packet_order == 1 ? c->rec.key : nullptr;   // 'direction': the launch writes the keys
    return r;
}

namespace {
__global__ void k_seq(int* v, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i] = (int)i;
}
}  // namespace

// The walk-order buffers of packet_order 'direction' for chunks of cap packets.
cudaError_t packet_order_alloc(mochii_ctx* c, long long cap) {
    RecordBuffers& r = c->rec;
    cudaError_t e;
    if ((e = cudaMalloc(&r.key, (size_t)cap * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&r.key_sorted, (size_t)cap * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&r.seq, (size_t)cap * 4)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&r.perm, (size_t)cap * 4)) != cudaSuccess) return e;
    r.sort_bytes = 0;
    if ((e = cub::DeviceRadixSort::SortPairs(nullptr, r.sort_bytes, r.key, r.key_sorted, r.seq, r.perm, (int)cap, 0,
                                             kCohKeyBits > kPacketKeyBits ? kCohKeyBits : kPacketKeyBits)) != cudaSuccess)
        return e;
    if ((e = cudaMalloc(&r.sort_tmp, r.sort_bytes + 16)) != cudaSuccess) return e;
    k_seq<<<grid_blocks(cap, 256, 148 * 16), 256, 0, c->stream>>>(r.seq, cap);
    return cudaGetLastError();
}

// The stellar packets of ionizing_field_and_rates (ionizing_field_mod.f90:
// 113-137), in chunks of the record buffer: launch, then walk.
cudaError_t launch_transport(mochii_ctx* c) {
    const PassArgs a = make_args(c);
    const PacketRecords r = packet_records(c);
    const int blocks = c->tw.ledger_blocks;
    for (long long ip0 = 0; ip0 < a.np; ip0 += r.cap) {
        const long long n = a.np - ip0 < r.cap ? a.np - ip0 : r.cap;
        const int lb = grid_blocks(n, kThreads, 1 << 30);
        const int acc = ip0 > 0;
        const bool amr = c->oct.ncells > 0;
        if (coherent_walk_applies(c)) {   // sort the chunk by coherent_key, launch and walk in that order
            k_coherent_keys<<<lb, kThreads, 0, c->stream>>>(a, ip0, n, c->rec.key);
            cudaError_t e = cub::DeviceRadixSort::SortPairs(c->rec.sort_tmp, c->rec.sort_bytes, c->rec.key,
                                                            c->rec.key_sorted, c->rec.seq, c->rec.perm, (int)n, 0,
                                                            kCohKeyBits, c->stream);
            if (e != cudaSuccess) return e;
            PacketRecords rl = r;
            rl.key = nullptr;
            rl.order = c->rec.perm;
            if (c->fp32) k_launch<float, false><<<lb, kThreads, 0, c->stream>>>(a, rl, ip0, n);
            else k_launch<double, false><<<lb, kThreads, 0, c->stream>>>(a, rl, ip0, n);
            WalkLaunch wl{n, ip0, acc, blocks, 0};
            wl.coherent = true;
            e = launch_walk_variant(c, a, r, wl);
            if (e != cudaSuccess) return e;
            continue;
        }
        if (c->fp32) {
            if (amr) k_launch<float, true><<<lb, kThreads, 0, c->stream>>>(a, r, ip0, n);
            else k_launch<float, false><<<lb, kThreads, 0, c->stream>>>(a, r, ip0, n);
        } else {
            if (amr) k_launch<double, true><<<lb, kThreads, 0, c->stream>>>(a, r, ip0, n);
            else k_launch<double, false><<<lb, kThreads, 0, c->stream>>>(a, r, ip0, n);
        }
        PacketRecords rw = r;
        if (r.key) {   // walk the chunk's packets in (source, direction) order
            cudaError_t e = cub::DeviceRadixSort::SortPairs(c->rec.sort_tmp, c->rec.sort_bytes, c->rec.key,
                                                            c->rec.key_sorted, c->rec.seq, c->rec.perm, (int)n, 0,
                                                            kPacketKeyBits, c->stream);
            if (e != cudaSuccess) return e;
            rw.perm = c->rec.perm;
        }
        const cudaError_t e = launch_walk_variant(c, a, rw, WalkLaunch{n, ip0, acc, blocks, 0, false});
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

// The diffuse packets (ionizing_field_mod.f90:139-161): their launch records
// come from launch_diffuse_chunk, the walk is the stellar one.  Under
// packet_order 'coherent' each chunk is sorted by diffuse_coherent_key and
// launched and walked (k_walk_coh) in that order, as the stellar chunks are.
cudaError_t launch_transport_diffuse(mochii_ctx* c, double total, long long nd) {
    const PassArgs a = make_args(c);
    const PacketRecords r = packet_records(c);
    const int blocks = c->tw.ledger_blocks;
    for (long long ip0 = 0; ip0 < nd; ip0 += r.cap) {
        const long long n = nd - ip0 < r.cap ? nd - ip0 : r.cap;
        if (coherent_walk_applies(c)) {
            cudaError_t e = launch_diffuse_keys(c, total, ip0, n, c->rec.key);
            if (e != cudaSuccess) return e;
            e = cub::DeviceRadixSort::SortPairs(c->rec.sort_tmp, c->rec.sort_bytes, c->rec.key, c->rec.key_sorted,
                                                c->rec.seq, c->rec.perm, (int)n, 0, kCohKeyBits, c->stream);
            if (e != cudaSuccess) return e;
            if ((e = launch_diffuse_chunk(c, total, ip0, n, c->rec.perm)) != cudaSuccess) return e;
            WalkLaunch wl{n, ip0, 1, blocks, 1};
            wl.coherent = true;
            if ((e = launch_walk_variant(c, a, r, wl)) != cudaSuccess) return e;
            continue;
        }
        cudaError_t e = launch_diffuse_chunk(c, total, ip0, n);
        if (e != cudaSuccess) return e;
        e = launch_walk_variant(c, a, r, WalkLaunch{n, ip0, 1, blocks, 1, false});
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}

cudaError_t launch_rates(mochii_ctx* c) {
    const double d2 = c->par.distance2cm * c->par.distance2cm;
    const double4* lg = c->oct.ncells > 0 ? c->oct.lgeo : nullptr;   // octree: per-leaf volume
    const double w = c->grid.dcell;
    const double fac = lg ? 1.0 : 1.0 / ((w * w * w) * d2);
    const double Lp = c->band.ion_Ltot / (double)c->par.nphotons;
    const double cg = Lp * 1.0e-18 / kEv2erg * fac;
    const double ch = Lp * 1.0e-18 * fac;
    const long long n = c->grid.nleaf;
    const int blocks = grid_blocks(n, 256, 148 * 16);
    const double* rk = c->rhokap;
    const double dc = c->par.distance2cm;
#define RATES(T, NT) k_rates<T, NT><<<blocks, 256, 0, c->stream>>>((const T*)c->tally, c->rates, n, cg, ch, lg, d2, rk, dc)
    if (c->fp32 && !c->tally64) {
        if (c->ntally == 2) RATES(float2, 2);
        else if (c->ntally == 6) RATES(float2, 6);
        else RATES(float2, 8);
    } else {
        if (c->ntally == 2) RATES(double, 2);
        else if (c->ntally == 6) RATES(double, 6);
        else RATES(double, 8);
    }
#undef RATES
    if (c->metal.ntr > 0 && c->metal.nmb > 0) {
        const int mb = (int)std::min<long long>((n + kRtM - 1) / kRtM, 148LL * 8);
        const int N = 2 * c->metal.ntrp;
        const bool pairs = c->fp32 && !c->tally64;
#define MOM(NU, KC)                                                                                              \
    do {                                                                                                         \
        if (c->metal.mom32)                                                                                      \
            k_metal_rates_mom<float, NU, KC, 8><<<mb, kRtThreads, 0, c->stream>>>(c->metal, n, cg, ch, lg, d2);  \
        else if (pairs)                                                                                          \
            k_metal_rates_mom<float2, NU, KC, kMomDeg><<<mb, kRtThreads, 0, c->stream>>>(c->metal, n, cg, ch, lg, d2); \
        else                                                                                                     \
            k_metal_rates_mom<double, NU, KC, kMomDeg><<<mb, kRtThreads, 0, c->stream>>>(c->metal, n, cg, ch, lg, d2); \
    } while (0)
        if (N <= 32) MOM(2, 32);
        else if (N <= 64) MOM(4, 32);
        else MOM(8, 16);
#undef MOM
    } else if (c->metal.ntr > 0) {
        const int mb = grid_blocks(n * c->metal.ntr, 256, 148 * 16);
        if (c->metal.raw32) k_metal_rates<float><<<mb, 256, 0, c->stream>>>(c->metal, n, cg, ch, lg, d2);
        else if (c->fp32 && !c->tally64) k_metal_rates<float2><<<mb, 256, 0, c->stream>>>(c->metal, n, cg, ch, lg, d2);
        else k_metal_rates<double><<<mb, 256, 0, c->stream>>>(c->metal, n, cg, ch, lg, d2);
    }
    return cudaGetLastError();
}

cudaError_t launch_jt_export(mochii_ctx* c, double* dst) {
    const long long n = c->grid.nleaf * (long long)c->nnu;
    const double Lp = c->band.ion_Ltot / (double)c->par.nphotons;
    const int blocks = grid_blocks(n, 256, 148 * 16);
    if (c->fp32 && !c->tally64) k_jt<float2><<<blocks, 256, 0, c->stream>>>((const float2*)c->jt, dst, n, Lp);
    else k_jt<double><<<blocks, 256, 0, c->stream>>>((const double*)c->jt, dst, n, Lp);
    return cudaGetLastError();
}

cudaError_t launch_sobol(const QmcTables* t, int stream01, long long idx0, long long n, int nd, double* out,
                         cudaStream_t s) {
    k_sobol<<<grid_blocks(n, 256, 148 * 16), 256, 0, s>>>(t, stream01, idx0, n, nd, out);
    return cudaGetLastError();
}

cudaError_t launch_walk(mochii_ctx* c, const double* rays, long long nray, int max_steps, int* leaves, int* nsteps) {
    if (c->oct.ncells > 0) {
        k_walk_amr_leaves<<<grid_blocks(nray, 128, 1 << 20), 128, 0, c->stream>>>(rays, nray, max_steps, leaves,
                                                                                 nsteps, c->oct);
        return cudaGetLastError();
    }
    k_walk<<<grid_blocks(nray, 128, 1 << 20), 128, 0, c->stream>>>(rays, nray, max_steps, leaves, nsteps,
                                                                     c->grid.xmin, c->grid.ymin, c->grid.zmin,
                                                                     c->grid.dcell, c->grid.nx, c->grid.ny, c->grid.nz);
    return cudaGetLastError();
}

cudaError_t launch_philox(uint64_t seed, uint32_t stream, uint64_t packet, int n0, int n, double* out) {
    k_philox<<<1, 32>>>(seed, stream, packet, n0, n, out);
    return cudaGetLastError();
}

cudaError_t launch_records(mochii_ctx* c, long long ip0, long long n, double* out) {
    const PassArgs a = make_args(c);
    k_launch_records<<<grid_blocks(n, 128, 1 << 20), 128, 0, c->stream>>>(a, ip0, n, out);
    return cudaGetLastError();
}

}  // namespace mochii

// ===========================================================================
// Launch records without allocation.
//
// mochii_launch_records stages the device-side records in a buffer it takes
// from cudaMallocAsync.  Some callers of this library cannot allocate device
// memory at call time: a host program whose device memory is handed out by
// another allocator (a PyTorch caching allocator, a Fortran host's memory
// pool, an MPS client under a memory limit) can see cudaMalloc fail although
// the job has room, and a time-critical loop may not accept an allocation.
// mochii_launch_records_noalloc stages the records in the file-scope device
// array below instead and calls no allocating routine.
//
// The array lives in every GPU that loads the library until the process
// exits (kNoallocMaxRecords x 8 doubles = 4 MiB).  Host code cannot use the
// array's name as a device address: each device's address is obtained once,
// with that device current, by cudaGetSymbolAddress on the first call made on
// that device (so make that first call before any stream capture).  Every
// call shares the array and it keeps the previous call's contents; the kernel
// writes every slot it reads back, so nothing has to start at zero.  Calls
// whose work overlaps on the GPU (several streams, several host threads)
// race on the array.
// ===========================================================================
namespace mochii {
namespace {
constexpr long long kNoallocMaxRecords = 65536;
static __device__ __align__(256) double g_noalloc_records[kNoallocMaxRecords * 8];

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kNoallocMaxDevices] = {};

// Device address of g_noalloc_records on the current device (set-up on the
// first call per device).
cudaError_t noalloc_scratch(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kNoallocMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_records);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
}
}  // namespace

long long noalloc_max_records() { return kNoallocMaxRecords; }

}  // namespace mochii

namespace mochii {
namespace {
// Dump of packet records for the test hooks: start cell, tMax, the H I
// cross section and the bin, as (ix, iy, iz, tMax_x, tMax_y, tMax_z,
// sigma_HI*1e18, inu); on the octree (leaf, -1, -1, x, y, z, sigma_HI*1e18,
// inu).
template <typename R>
__global__ void k_records_dump(const PacketRecords r, long long n, double* out, int amr) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int cell = r.cell[i];
    double* o = out + 8 * i;
    if (amr) {
        o[0] = cell; o[1] = -1.0; o[2] = -1.0;
    } else {
        o[0] = cell & 1023; o[1] = (cell >> 10) & 1023; o[2] = (cell >> 20) & 1023;
    }
    o[3] = r.tm[i]; o[4] = r.tm[r.cap + i]; o[5] = r.tm[2 * r.cap + i];
    o[6] = (double)static_cast<const R*>(r.sig)[i];
    o[7] = (double)(r.bits[i] & 0xFFFF);
}
}  // namespace

cudaError_t launch_records_from_buffer(mochii_ctx* c, long long n, double* host_out) {
    double* d = nullptr;
    cudaError_t e = cudaMallocAsync(&d, (size_t)n * 64, c->stream);
    if (e != cudaSuccess) return e;
    const PacketRecords r = packet_records(c);
    const int amr = c->oct.ncells > 0;
    if (c->fp32) k_records_dump<float><<<grid_blocks(n, 128, 1 << 30), 128, 0, c->stream>>>(r, n, d, amr);
    else k_records_dump<double><<<grid_blocks(n, 128, 1 << 30), 128, 0, c->stream>>>(r, n, d, amr);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_out, d, (size_t)n * 64, cudaMemcpyDeviceToHost, c->stream);
    cudaFreeAsync(d, c->stream);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(c->stream);
}

cudaError_t launch_records_noalloc(mochii_ctx* c, long long ip0, long long n, double* host_out) {
    double* scratch = nullptr;
    cudaError_t e = noalloc_scratch(&scratch);
    if (e != cudaSuccess) return e;
    const PassArgs a = make_args(c);
    k_launch_records<<<grid_blocks(n, 128, 1 << 20), 128, 0, c->stream>>>(a, ip0, n, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(host_out, scratch, (size_t)n * 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(c->stream);
}

}  // namespace mochii
