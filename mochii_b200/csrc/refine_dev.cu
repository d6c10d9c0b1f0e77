// Device plan of the I-front re-refinement (amr_refine_mod.f90:46-436) for a
// context on an octree.  The same plan as the host's (refine.cpp), restated
// for one thread per item:
//
//   k_front   front flags, one thread per old leaf: eps < x_HI < 1 - eps, or
//             a face-neighbour gas leaf (the leaf across the face) differing
//             by more than dx (:66-88)
//   k_level   one thread per cell of the current level: split when the level
//             is below refine_lbase, or below refine_lmax with a front leaf
//             overlapping the cell (cell_has_front, :398-422, a bounded
//             descent of the old tree); a kept cell becomes a new leaf, a
//             split one its 8 children of the next level (rec_build,
//             :355-380)
//   sort      the new leaves into rec_build's depth-first order: a leaf's key
//             is its octant path (3 bits a level, ix + 2 iy + 4 iz) padded
//             to refine_lmax levels, and depth-first order is key order
//   k_remap   one thread per new leaf: the overlap-volume remap of remap_leaf
//             (:197-292) by a bounded descent of the old tree
//
// Each descent visits the old cells in the host plan's order and sums in
// the same order, so the plans agree to the bit.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include <cub/cub.cuh>

#include "ctx.h"
#include "octree.h"
#include "refine.h"

namespace mochii {

namespace {

constexpr int kStackDev = 512;   // as the host descents; 7 x depth + 1 entries at most
constexpr int kT = 256;

struct OldTree {
    const double4* geo;
    const int* children;
    const int* ileaf;
};

__global__ void k_front(const int* __restrict__ lnext, const double* __restrict__ nH, const double* __restrict__ xHI,
                        long long n, double eps, double dx, unsigned char* __restrict__ front) {
    const long long il = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (il >= n) return;
    unsigned char f = 0;
    if (nH[il] > 0.0) {
        const double xr = xHI[il];
        if (xr > eps && xr < 1.0 - eps) {
            f = 1;
        } else {
            for (int k = 0; k < 6; ++k) {
                const int jl = lnext[8 * il + k];   // the leaf across the face, < 0 none or finer
                if (jl < 0 || nH[jl] <= 0.0) continue;
                if (fabs(xHI[jl] - xr) > dx) {
                    f = 1;
                    break;
                }
            }
        }
    }
    front[il] = f;
}

__device__ bool has_front(const OldTree& t, const unsigned char* front, double x, double y, double z, double h,
                          int* ovf) {
    int stack[kStackDev];
    int n = 1;
    stack[0] = 0;
    while (n > 0) {
        const int c = stack[--n];
        const double4 g = t.geo[c];
        if (fabs(g.x - x) > g.w + h) continue;
        if (fabs(g.y - y) > g.w + h) continue;
        if (fabs(g.z - z) > g.w + h) continue;
        const int lf = t.ileaf[c];
        if (lf >= 0) {
            if (front[lf]) return true;
            continue;
        }
        for (int k = 0; k < 8; ++k) {
            const int j = t.children[8 * c + k];
            if (j < 0) continue;
            if (n >= kStackDev) {
                atomicExch(ovf, 1);
                return false;
            }
            stack[n++] = j;
        }
    }
    return false;
}

// Split decisions of the m cells of one level (half width h).
__global__ void k_split(OldTree t, const unsigned char* __restrict__ front, const double* __restrict__ cx,
                        const double* __restrict__ cy, const double* __restrict__ cz, long long m, int level, int lbase,
                        int lmax, double h, int* __restrict__ split, int* ovf) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const bool s = (level < lmax && has_front(t, front, cx[i], cy[i], cz[i], h, ovf)) || level < lbase;
    split[i] = s ? 1 : 0;
}

// Kept cells to the leaf chunk (at i - off[i]), split cells to their eight
// children (at 8 off[i] + octant) with the octant appended to the key.
__global__ void k_emit(const double* __restrict__ cx, const double* __restrict__ cy, const double* __restrict__ cz,
                       const unsigned long long* __restrict__ key, const int* __restrict__ split,
                       const int* __restrict__ off, long long m, double h, int shift, double* lx, double* ly,
                       double* lz, unsigned long long* lkey, double* nx, double* ny, double* nz,
                       unsigned long long* nkey) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    if (!split[i]) {
        const long long j = i - off[i];
        lx[j] = cx[i];
        ly[j] = cy[i];
        lz[j] = cz[i];
        lkey[j] = key[i];
        return;
    }
    const double hc = 0.5 * h;
    const long long b = 8LL * off[i];
    for (int o = 0; o < 8; ++o) {
        const int ix = o & 1, iy = (o >> 1) & 1, iz = o >> 2;
        nx[b + o] = cx[i] + (double)(2 * ix - 1) * hc;
        ny[b + o] = cy[i] + (double)(2 * iy - 1) * hc;
        nz[b + o] = cz[i] + (double)(2 * iz - 1) * hc;
        nkey[b + o] = key[i] | ((unsigned long long)o << shift);
    }
}

__device__ __forceinline__ double overlap_1d(double ca, double ha, double cb, double hb) {
    const double ov = fmin(ca + ha, cb + hb) - fmax(ca - ha, cb - hb);
    return ov < 0.0 ? 0.0 : ov;
}

struct OldState {
    const double *nH, *ne, *rk, *x1, *x2, *x3, *te;
    double yHe, te_min;
};

struct NewLeaves {
    const double *x, *y, *z;
    const int* lev;
    double* out;   // 7 x n: nH, n_e, rhokap, x_HI, x_HeI, x_HeII, T_e
    long long n;
};

__global__ void k_remap(OldTree t, OldState s, NewLeaves nl, double half, int* ovf) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nl.n) return;
    const double x = nl.x[i], y = nl.y[i], z = nl.z[i];
    const double h = half / ldexp(1.0, nl.lev[i]);
    double sv = 0, snh = 0, sne = 0, srk = 0, sm = 0, smx1 = 0, smx2 = 0, smx3 = 0, st = 0, ste = 0;
    double svx1 = 0, svx2 = 0, svx3 = 0, svte = 0;
    int stack[kStackDev];
    int n = 1;
    stack[0] = 0;
    bool over = false;
    while (n > 0) {
        const int c = stack[--n];
        const double4 g = t.geo[c];
        const double hw = g.w;
        if (fabs(g.x - x) >= hw + h) continue;
        if (fabs(g.y - y) >= hw + h) continue;
        if (fabs(g.z - z) >= hw + h) continue;
        const int jl = t.ileaf[c];
        if (jl >= 0) {
            const double ov = overlap_1d(g.x, hw, x, h) * overlap_1d(g.y, hw, y, h) * overlap_1d(g.z, hw, z, h);
            if (ov <= 0.0) continue;
            const double nh = s.nH[jl], ne = s.ne[jl];
            sv = sv + ov;
            snh = snh + nh * ov;
            sne = sne + ne * ov;
            srk = srk + (s.rk ? s.rk[jl] : 0.0) * ov;
            const double wm = nh * ov;
            sm = sm + wm;
            smx1 = smx1 + wm * s.x1[jl];
            smx2 = smx2 + wm * s.x2[jl];
            smx3 = smx3 + wm * s.x3[jl];
            const double wt = (nh * (1.0 + s.yHe) + ne) * ov;
            st = st + wt;
            ste = ste + wt * s.te[jl];
            svx1 = svx1 + ov * s.x1[jl];
            svx2 = svx2 + ov * s.x2[jl];
            svx3 = svx3 + ov * s.x3[jl];
            svte = svte + ov * s.te[jl];
            continue;
        }
        for (int k = 0; k < 8 && !over; ++k) {
            const int j = t.children[8 * c + k];
            if (j < 0) continue;
            if (n >= kStackDev) {
                over = true;
                break;
            }
            stack[n++] = j;
        }
        if (over) break;
    }
    if (over) atomicExch(ovf, 1);
    const double vol = (2.0 * h) * (2.0 * h) * (2.0 * h);
    double* o = nl.out;
    const long long N = nl.n;
    o[i] = snh / vol;
    o[N + i] = sne / vol;
    o[2 * N + i] = srk / vol;
    double a1, a2, a3;
    if (sm > 0.0) {
        a1 = smx1 / sm; a2 = smx2 / sm; a3 = smx3 / sm;
    } else if (sv > 0.0) {
        a1 = svx1 / sv; a2 = svx2 / sv; a3 = svx3 / sv;
    } else {
        a1 = 1.0; a2 = 1.0; a3 = 0.0;
    }
    o[3 * N + i] = a1;
    o[4 * N + i] = a2;
    o[5 * N + i] = a3;
    o[6 * N + i] = st > 0.0 ? ste / st : sv > 0.0 ? svte / sv : s.te_min;
}

__global__ void k_iota(int* v, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int)i;
}

__global__ void k_gather(const int* __restrict__ perm, const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ z, const int* __restrict__ lev, long long n, double* ox,
                         double* oy, double* oz, int* olev) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = perm[i];
    ox[i] = x[p];
    oy[i] = y[p];
    oz[i] = z[p];
    olev[i] = lev[p];
}

__global__ void k_fill_int(int* v, long long n, int value) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = value;
}

int blocks_for(long long n) { return (int)((n + kT - 1) / kT); }

// Device buffers released at scope end.
struct DevPool {
    std::vector<void*> p;
    template <typename T>
    cudaError_t get(T** out, size_t count) {
        void* q = nullptr;
        const cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 16);
        if (e == cudaSuccess) p.push_back(q);
        *out = static_cast<T*>(q);
        return e;
    }
    ~DevPool() {
        for (void* q : p) cudaFree(q);
    }
};

struct Chunk {
    double *x, *y, *z;
    unsigned long long* key;
    long long n;
    int level;
};

}  // namespace

bool refine_plan_device(mochii_ctx* c, const RefineIn& in, RefineOut& out, std::string* err) {
    auto failed = [&](const char* what, cudaError_t e) {
        if (err) *err = std::string("re-refinement on the device: ") + what + ": " + cudaGetErrorString(e);
        return false;
    };
    out = RefineOut();
    const long long nold = c->grid.nleaf;
    const cudaStream_t st = c->stream;
    const OldTree t{c->oct.geo, c->oct.children, c->oct.ileaf};
    const double half = c->oct.half;
    DevPool pool;
    cudaError_t e;
    unsigned char* front;
    int* ovf;
    if ((e = pool.get(&front, (size_t)nold)) || (e = pool.get(&ovf, 1))) return failed("allocation", e);
    if ((e = cudaMemsetAsync(ovf, 0, sizeof(int), st))) return failed("memset", e);
    k_front<<<blocks_for(nold), kT, 0, st>>>(c->oct.lnext, c->nH, c->xHI, nold, in.eps, in.dx, front);
    // level by level from the root
    std::vector<Chunk> chunks;
    long long m = 1;
    double *cx, *cy, *cz;
    unsigned long long* ck;
    if ((e = pool.get(&cx, 1)) || (e = pool.get(&cy, 1)) || (e = pool.get(&cz, 1)) || (e = pool.get(&ck, 1)))
        return failed("allocation", e);
    const double zero = 0.0;
    const unsigned long long kz0 = 0ULL;
    for (double* q : {cx, cy, cz})
        if ((e = cudaMemcpyAsync(q, &zero, sizeof(double), cudaMemcpyHostToDevice, st))) return failed("copy", e);
    if ((e = cudaMemcpyAsync(ck, &kz0, sizeof(kz0), cudaMemcpyHostToDevice, st))) return failed("copy", e);
    for (int level = 0; m > 0; ++level) {
        const double h = half / std::ldexp(1.0, level);
        int *split, *off;
        if ((e = pool.get(&split, (size_t)m)) || (e = pool.get(&off, (size_t)m))) return failed("allocation", e);
        k_split<<<blocks_for(m), kT, 0, st>>>(t, front, cx, cy, cz, m, level, in.lbase, in.lmax, h, split, ovf);
        size_t tmp_bytes = 0;
        if ((e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, split, off, (int)m, st))) return failed("scan", e);
        char* tmp;
        if ((e = pool.get(&tmp, tmp_bytes))) return failed("allocation", e);
        if ((e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, split, off, (int)m, st))) return failed("scan", e);
        int last_off = 0, last_split = 0;
        if ((e = cudaMemcpyAsync(&last_off, off + m - 1, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
            (e = cudaMemcpyAsync(&last_split, split + m - 1, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
            (e = cudaStreamSynchronize(st)))
            return failed("level count", e);
        const long long nsplit = (long long)last_off + last_split;
        const long long nkeep = m - nsplit;
        if (8 * nsplit + nkeep > (long long)2000000000) {
            if (err) *err = "re-refinement on the device: more than 2e9 cells in one level";
            return false;
        }
        Chunk ch{nullptr, nullptr, nullptr, nullptr, nkeep, level};
        double *nx = nullptr, *ny = nullptr, *nz = nullptr;
        unsigned long long* nk = nullptr;
        if ((e = pool.get(&ch.x, (size_t)nkeep)) || (e = pool.get(&ch.y, (size_t)nkeep)) ||
            (e = pool.get(&ch.z, (size_t)nkeep)) || (e = pool.get(&ch.key, (size_t)nkeep)) ||
            (e = pool.get(&nx, (size_t)(8 * nsplit))) || (e = pool.get(&ny, (size_t)(8 * nsplit))) ||
            (e = pool.get(&nz, (size_t)(8 * nsplit))) || (e = pool.get(&nk, (size_t)(8 * nsplit))))
            return failed("allocation", e);
        const int shift = 3 * (in.lmax - (level + 1));   // used only when a cell splits (level < lmax)
        k_emit<<<blocks_for(m), kT, 0, st>>>(cx, cy, cz, ck, split, off, m, h, shift < 0 ? 0 : shift, ch.x, ch.y,
                                            ch.z, ch.key, nx, ny, nz, nk);
        if (nkeep > 0) chunks.push_back(ch);
        cx = nx; cy = ny; cz = nz; ck = nk;
        m = 8 * nsplit;
        if (level > in.lmax) break;   // nothing splits at refine_lmax
    }
    long long N = 0;
    for (const Chunk& ch : chunks) N += ch.n;
    if (N <= 0 || N > (long long)2000000000) {
        if (err) *err = "re-refinement on the device: no new leaves or too many";
        return false;
    }
    // gather the chunks, sort by the depth-first key
    double *ax, *ay, *az, *sx, *sy, *sz;
    int *alev, *slev, *idx, *perm;
    unsigned long long *akey, *skey;
    if ((e = pool.get(&ax, N)) || (e = pool.get(&ay, N)) || (e = pool.get(&az, N)) || (e = pool.get(&alev, N)) ||
        (e = pool.get(&akey, N)) || (e = pool.get(&skey, N)) || (e = pool.get(&idx, N)) || (e = pool.get(&perm, N)) ||
        (e = pool.get(&sx, N)) || (e = pool.get(&sy, N)) || (e = pool.get(&sz, N)) || (e = pool.get(&slev, N)))
        return failed("allocation", e);
    long long at = 0;
    for (const Chunk& ch : chunks) {
        const size_t b8 = (size_t)ch.n * 8;
        if ((e = cudaMemcpyAsync(ax + at, ch.x, b8, cudaMemcpyDeviceToDevice, st)) ||
            (e = cudaMemcpyAsync(ay + at, ch.y, b8, cudaMemcpyDeviceToDevice, st)) ||
            (e = cudaMemcpyAsync(az + at, ch.z, b8, cudaMemcpyDeviceToDevice, st)) ||
            (e = cudaMemcpyAsync(akey + at, ch.key, b8, cudaMemcpyDeviceToDevice, st)))
            return failed("gather", e);
        k_fill_int<<<blocks_for(ch.n), kT, 0, st>>>(alev + at, ch.n, ch.level);
        at += ch.n;
    }
    k_iota<<<blocks_for(N), kT, 0, st>>>(idx, N);
    {
        size_t tmp_bytes = 0;
        const int bits = 3 * in.lmax;
        if ((e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, akey, skey, idx, perm, (int)N, 0, bits, st)))
            return failed("sort", e);
        char* tmp;
        if ((e = pool.get(&tmp, tmp_bytes))) return failed("allocation", e);
        if ((e = cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, akey, skey, idx, perm, (int)N, 0, bits, st)))
            return failed("sort", e);
    }
    k_gather<<<blocks_for(N), kT, 0, st>>>(perm, ax, ay, az, alev, N, sx, sy, sz, slev);
    // remap
    double* rout;
    if ((e = pool.get(&rout, 7 * (size_t)N))) return failed("allocation", e);
    const OldState os{c->nH, c->ne, c->rhokap, c->xHI, c->xHeI, c->xHeII, c->Te, in.yHe, in.te_min};
    k_remap<<<blocks_for(N), kT, 0, st>>>(t, os, NewLeaves{sx, sy, sz, slev, rout, N}, half, ovf);
    if ((e = cudaGetLastError())) return failed("launch", e);
    // results to the host
    std::vector<unsigned char> fr((size_t)nold);
    int over = 0;
    out.x.resize(N); out.y.resize(N); out.z.resize(N); out.lev.resize(N);
    out.nH.resize(N); out.ne.resize(N); out.rk.resize(N); out.x1.resize(N); out.x2.resize(N); out.x3.resize(N);
    out.te.resize(N);
    std::vector<double>* cols[7] = {&out.nH, &out.ne, &out.rk, &out.x1, &out.x2, &out.x3, &out.te};
    if ((e = cudaMemcpyAsync(fr.data(), front, (size_t)nold, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(&over, ovf, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(out.x.data(), sx, (size_t)N * 8, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(out.y.data(), sy, (size_t)N * 8, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(out.z.data(), sz, (size_t)N * 8, cudaMemcpyDeviceToHost, st)) ||
        (e = cudaMemcpyAsync(out.lev.data(), slev, (size_t)N * 4, cudaMemcpyDeviceToHost, st)))
        return failed("copy back", e);
    for (int k = 0; k < 7; ++k)
        if ((e = cudaMemcpyAsync(cols[k]->data(), rout + (size_t)k * N, (size_t)N * 8, cudaMemcpyDeviceToHost, st)))
            return failed("copy back", e);
    if ((e = cudaStreamSynchronize(st))) return failed("synchronise", e);
    if (over) {
        if (err) *err = "re-refinement: octree descent stack overflow";
        return false;
    }
    for (unsigned char f : fr) out.nfront += f;
    return true;
}

}  // namespace mochii
