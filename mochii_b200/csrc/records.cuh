// Packet records: the hand-off between the launch kernels (stellar and
// diffuse) and the walk kernel.  Structure of arrays over the packets of one
// chunk: the DDA state after dda_init (tMax, tDelta, start cell, step
// signs), the diagnostic bin, and the packet's cross sections and
// rate coefficients at its exact energy.
#pragma once
#include <cuda_runtime.h>

#include "dust.cuh"
#include "physics.cuh"

namespace mochii {

// Record bits above the bin and DDA steps: an external-field packet
// (photon%from_external) and its entry surface, 0-5 the box face
// (+x, -x, +y, -y, +z, -z), 6 the sphere.
constexpr int kExternalBit = 1 << 22;
constexpr int kExternalFaceShift = 23;

struct PacketRecords {
    double* tm;    // 3 x cap (octree: start point)
    double* td;    // 3 x cap (octree: direction)
    int* cell;     // ix | iy << 10 | iz << 20 (octree: start leaf, -1 outside)
    int* bits;     // inu | (stp_x+1) << 16 | (stp_y+1) << 18 | (stp_z+1) << 20 (octree: inu),
                   // + kExternalBit | face << kExternalFaceShift for external packets
    void* sig;     // 3 x cap of R: sigma_HI, sigma_HeI, sigma_HeII in 1e-18 cm^2
                   // (+ a 4th row with grains or FUV: the dust extinction coefficient)
    void* coef;    // 6 x cap of R: Gamma/heat coefficients per unit path
                   // (+ rows 6, 7 with grains or FUV: dust absorption coefficient, E < eion_min)
    double* E;     // metals only: packet energy [eV]
    void* msig;    // metals only: ntrp x cap of R, active-prefix sigma_k in 1e-18 cm^2
    void* dsc;     // scattering only: 2 x cap of R, dust scattering coefficient and <cos>
    double* p0;    // scattering on the Cartesian grid: start point and direction, 6 x cap
    long long cap;
    unsigned* key = nullptr;     // packet_order 'direction': source and direction cell of each packet
    const int* perm = nullptr;   // walk order (the chunk's packets by key), null: launch order
    const int* order = nullptr;  // packet_order 'coherent': record t holds chunk packet order[t]
};

// Walk-order key of packet_order 'coherent', from the packet's launch
// uniforms alone (so the chunk can be sorted before its records exist):
// source component (4 bits), a direction cell of 64 equal-area bands in
// cos(theta) x 128 sectors in phi, the sectors of odd bands reversed so that
// consecutive cells are neighbours on the sphere (13 bits), and the energy
// quantile of the source spectrum in 256 steps (8 bits).  Packets of one
// warp then leave in nearly the same direction with nearly the same energy,
// so they cross the same leaves and score the same spectrum and moment bins.
constexpr int kCohKeyBits = 25;
__device__ __forceinline__ unsigned coherent_key(int ic, double umu, double uphi, double ue) {
    const unsigned band = (unsigned)min((int)(umu * 64.0), 63);
    unsigned sec = (unsigned)min((int)(uphi * 128.0), 127);
    if (band & 1u) sec = 127u - sec;
    const unsigned eq = (unsigned)min((int)(ue * 256.0), 255);
    return ((unsigned)(ic & 15) << 21) | (((band << 7) | sec) << 8) | eq;
}

// Walk-order key of a diffuse packet under packet_order 'coherent', from
// its launch uniforms and start cell: a direction cell of 32 equal-area
// bands in cos(theta) x 32 sectors in phi, the sectors of odd bands
// reversed (10 bits), above the Morton code of the start cell on a 32^3
// coarsening of the grid (15 bits).  Packets of one warp then leave nearly
// parallel from one neighbourhood, so their walks stay together and end
// together.  Fits the kCohKeyBits of the stellar key.
__device__ __forceinline__ unsigned diffuse_coherent_key(double umu, double uphi, int ix, int iy, int iz,
                                                         const int* n) {
    const unsigned band = (unsigned)min((int)(umu * 32.0), 31);
    unsigned sec = (unsigned)min((int)(uphi * 32.0), 31);
    if (band & 1u) sec = 31u - sec;
    const unsigned cx = (unsigned)min((ix * 32) / n[0], 31), cy = (unsigned)min((iy * 32) / n[1], 31),
                   cz = (unsigned)min((iz * 32) / n[2], 31);
    unsigned m = 0;
#pragma unroll
    for (int b = 0; b < 5; ++b)
        m |= (((cx >> b) & 1u) << (3 * b)) | (((cy >> b) & 1u) << (3 * b + 1)) | (((cz >> b) & 1u) << (3 * b + 2));
    return (((band << 5) | sec) << 15) | m;
}

constexpr int kPacketKeyBits = 18;

// Walk-order key of a stellar packet: source component (3 bits), direction
// octant (3 bits) and a 64 x 64 cell of (|k_x|, |k_y|) in the octant,
// Morton-interleaved so nearby directions get nearby keys.
__device__ __forceinline__ unsigned packet_dir_key(int ic, const double* kk) {
    const unsigned oct = (kk[0] < 0.0 ? 1u : 0u) | (kk[1] < 0.0 ? 2u : 0u) | (kk[2] < 0.0 ? 4u : 0u);
    const unsigned qx = (unsigned)min((int)(fabs(kk[0]) * 64.0), 63), qy = (unsigned)min((int)(fabs(kk[1]) * 64.0), 63);
    unsigned m = 0;
#pragma unroll
    for (int b = 0; b < 6; ++b) m |= (((qx >> b) & 1u) << (2 * b)) | (((qy >> b) & 1u) << (2 * b + 1));
    return ((unsigned)(ic & 7) << 15) | (oct << 12) | m;
}

template <typename R>
__device__ __forceinline__ void write_cross_sections(const PacketRecords& rec, long long i, double E) {
    const double sHI = sigma_HI(E), sHeI = sigma_HeI(E), sHeII = sigma_HeII(E);
    R* sg = static_cast<R*>(rec.sig);
    R* cf = static_cast<R*>(rec.coef);
    const long long c = rec.cap;
    sg[i] = (R)(sHI * 1.0e18);
    sg[c + i] = (R)(sHeI * 1.0e18);
    sg[2 * c + i] = (R)(sHeII * 1.0e18);
    cf[i] = (R)(sHI * 1.0e18 / E);
    cf[c + i] = (R)(sHI * 1.0e18 * fmax(1.0 - kEthHI / E, 0.0));
    cf[2 * c + i] = (R)(sHeI * 1.0e18 / E);
    cf[3 * c + i] = (R)(sHeI * 1.0e18 * fmax(1.0 - kEthHeI / E, 0.0));
    cf[4 * c + i] = (R)(sHeII * 1.0e18 / E);
    cf[5 * c + i] = (R)(sHeII * 1.0e18 * fmax(1.0 - kEthHeII / E, 0.0));
}

// The grain and FUV part of a packet record (build_ion_packet_physics
// dust cache, ion_packet_mod.f90:42-50; score_ion_path dust_abs_path and
// fuv_field_path terms, ion_score_mod.f90:163-166,206-209): the extinction
// coefficient the walk multiplies with rhokap (absorption, plus scattering
// when scattering is on), the absorption coefficient it scores, whether the
// packet is an FUV packet, and for the scattered flights the scattering
// coefficient, <cos> and (Cartesian grid) the start point and direction.
template <typename R>
__device__ __forceinline__ void write_grain_record(const PacketRecords& rec, long long i, const DustDev& d,
                                                   int scatter, double eion_min, double E, const double pos[3],
                                                   const double kk[3], int car) {
    const long long c = rec.cap;
    DustOptics o = {0.0, 0.0, 0.0};
    if (d.n > 0) o = dust_optics(d, E);
    static_cast<R*>(rec.sig)[3 * c + i] = (R)(scatter ? o.sabs + o.ssca : o.sabs);
    R* cf = static_cast<R*>(rec.coef);
    cf[6 * c + i] = (R)o.sabs;
    cf[7 * c + i] = E < eion_min ? (R)1 : (R)0;
    if (scatter) {
        R* ds = static_cast<R*>(rec.dsc);
        ds[i] = (R)o.ssca;
        ds[c + i] = (R)o.g;
    }
}

// Record of one packet on the octree: the cross sections, start point,
// direction and start leaf (the walk finds its faces as it goes).
template <typename R>
__device__ __forceinline__ void write_record_amr(const PacketRecords& rec, long long i, const double pos[3],
                                                 const double kk[3], double E, int inu, int leaf) {
    write_cross_sections<R>(rec, i, E);
    const long long c = rec.cap;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        rec.tm[k * c + i] = pos[k];
        rec.td[k * c + i] = kk[k];
    }
    rec.cell[i] = leaf;
    rec.bits[i] = inu;
}

// Record of one packet: build_ion_packet_physics (ion_packet_mod.f90:21-53),
// the per-path coefficients of score_ion_path (ion_score_mod.f90:213-221),
// scaled by 1e18 so FP32 stays in range (sigma in 1e-18 cm^2, E in eV), and
// dda_init (raytrace_amr.f90:495-532) in FP64.
template <typename R>
__device__ __forceinline__ void write_record(const PacketRecords& rec, long long i, const double pos[3],
                                             const double kk[3], double E, int inu, const double org[3],
                                             double d, const int n[3]) {
    write_cross_sections<R>(rec, i, E);
    const long long c = rec.cap;
    int idx[3], bits = inu;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        idx[k] = min(max((int)((pos[k] - org[k]) / d), 0), n[k] - 1);
        double tmv, tdv;
        int st;
        if (kk[k] > 0.0) {
            st = 1; tmv = (org[k] + (double)(idx[k] + 1) * d - pos[k]) / kk[k]; tdv = d / kk[k];
        } else if (kk[k] < 0.0) {
            st = -1; tmv = (org[k] + (double)idx[k] * d - pos[k]) / kk[k]; tdv = -d / kk[k];
        } else {
            st = 0; tmv = kHugest; tdv = kHugest;
        }
        rec.tm[k * c + i] = tmv;
        rec.td[k * c + i] = tdv;
        bits |= (st + 1) << (16 + 2 * k);
    }
    rec.cell[i] = idx[0] | (idx[1] << 10) | (idx[2] << 20);
    rec.bits[i] = bits;
    if (rec.p0) {   // start point and direction: scattered flights and peel-off
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            rec.p0[k * c + i] = pos[k];
            rec.p0[(3 + k) * c + i] = kk[k];
        }
    }
}

}  // namespace mochii
