// Solution-driven I-front re-refinement of the octree (amr_refine_mod.f90).
//
// The reference rebuilds its octree in place between two iterations
// (main.f90:172-178).  Here every leaf-indexed buffer of a context (state,
// columns, tallies, records, metal arrays, octree tables) is sized by the
// leaf count, so a rebuilt tree is a new context: the plan is host work --
// flag the front leaves, build the new leaf list, remap the state by overlap
// volume, check the conserved box integrals -- the new leaf list (with the
// remapped state as extra columns) goes to a file, and mochii_refine_front
// initialises a context from it and sets the remapped state.
//
//   front      a gas leaf with eps < x_HI < 1 - eps (par%refine_eps), or whose
//              face neighbour (a gas leaf) differs by more than par%refine_dx
//              in x_HI (:66-88)
//   new tree   level par%refine_lmax wherever a cell overlaps a front leaf,
//              par%refine_lbase elsewhere (rec_build, cell_has_front,
//              :355-422)
//   remap      nH, n_e, rhokap by volume; x_HI, x_HeI, x_HeII by nH V; T_e by
//              (nH (1 + He/H) + n_e) V; plain volume averages where a region
//              holds no material (remap_leaf, :197-292)
//   check      the box integrals of H nuclei, H I, He I, He II, electrons,
//              extinction and thermal content before and after agree to 1e-8
//              (conservation_report, :299-352)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <charconv>

#include "ctx.h"
#include "mochii_gpu.h"
#include "octree.h"
#include "refine.h"

namespace mochii {

namespace {

constexpr int kStack = 512;   // the descents' explicit stack (:209)

double overlap_1d(double ca, double ha, double cb, double hb) {
    const double ov = std::min(ca + ha, cb + hb) - std::max(ca - ha, cb - hb);
    return ov < 0.0 ? 0.0 : ov;
}

struct Planner {
    const OctHost& o;
    const RefineIn& in;
    std::vector<char> front;
    RefineOut& out;
    bool overflow = false;

    double cx(int c) const { return o.geo[4 * (size_t)c]; }
    double cy(int c) const { return o.geo[4 * (size_t)c + 1]; }
    double cz(int c) const { return o.geo[4 * (size_t)c + 2]; }
    double ch(int c) const { return o.geo[4 * (size_t)c + 3]; }

    // cell_has_front (:398-422): does the cell overlap a front leaf?
    bool has_front(double x, double y, double z, double h) {
        int stack[kStack], n = 1;
        stack[0] = 0;
        while (n > 0) {
            const int c = stack[--n];
            if (std::fabs(cx(c) - x) > ch(c) + h) continue;
            if (std::fabs(cy(c) - y) > ch(c) + h) continue;
            if (std::fabs(cz(c) - z) > ch(c) + h) continue;
            if (o.ileaf[c] >= 0) {
                if (front[o.ileaf[c]]) return true;
                continue;
            }
            for (int k = 0; k < 8; ++k) {
                const int j = o.children[8 * (size_t)c + k];
                if (j < 0) continue;
                if (n >= kStack) { overflow = true; return false; }
                stack[n++] = j;
            }
        }
        return false;
    }

    // rec_build (:355-380): depth first, octants ix + 2 iy + 4 iz.
    void build(double x, double y, double z, double h, int level) {
        if ((level < in.lmax && has_front(x, y, z, h)) || level < in.lbase) {
            const double hc = 0.5 * h;
            for (int iz = 0; iz < 2; ++iz)
                for (int iy = 0; iy < 2; ++iy)
                    for (int ix = 0; ix < 2; ++ix)
                        build(x + (double)(2 * ix - 1) * hc, y + (double)(2 * iy - 1) * hc,
                              z + (double)(2 * iz - 1) * hc, hc, level + 1);
        } else {
            out.x.push_back(x);
            out.y.push_back(y);
            out.z.push_back(z);
            out.lev.push_back(level);
        }
    }

    // remap_leaf (:197-292).
    void remap(double x, double y, double z, double h) {
        double sv = 0, snh = 0, sne = 0, srk = 0, sm = 0, smx1 = 0, smx2 = 0, smx3 = 0, st = 0, ste = 0;
        double svx1 = 0, svx2 = 0, svx3 = 0, svte = 0;
        int stack[kStack], n = 1;
        stack[0] = 0;
        while (n > 0) {
            const int c = stack[--n];
            const double hw = ch(c);
            if (std::fabs(cx(c) - x) >= hw + h) continue;
            if (std::fabs(cy(c) - y) >= hw + h) continue;
            if (std::fabs(cz(c) - z) >= hw + h) continue;
            const int jl = o.ileaf[c];
            if (jl >= 0) {
                const double ov = overlap_1d(cx(c), hw, x, h) * overlap_1d(cy(c), hw, y, h) *
                                  overlap_1d(cz(c), hw, z, h);
                if (ov <= 0.0) continue;
                sv = sv + ov;
                snh = snh + in.nH[jl] * ov;
                sne = sne + in.ne[jl] * ov;
                srk = srk + (in.rk ? in.rk[jl] : 0.0) * ov;
                const double wm = in.nH[jl] * ov;
                sm = sm + wm;
                smx1 = smx1 + wm * in.xHI[jl];
                smx2 = smx2 + wm * in.xHeI[jl];
                smx3 = smx3 + wm * in.xHeII[jl];
                const double wt = (in.nH[jl] * (1.0 + in.yHe) + in.ne[jl]) * ov;
                st = st + wt;
                ste = ste + wt * in.Te[jl];
                svx1 = svx1 + ov * in.xHI[jl];
                svx2 = svx2 + ov * in.xHeI[jl];
                svx3 = svx3 + ov * in.xHeII[jl];
                svte = svte + ov * in.Te[jl];
                continue;
            }
            for (int k = 0; k < 8; ++k) {
                const int j = o.children[8 * (size_t)c + k];
                if (j < 0) continue;
                if (n >= kStack) { overflow = true; return; }
                stack[n++] = j;
            }
        }
        const double vol = (2.0 * h) * (2.0 * h) * (2.0 * h);
        out.nH.push_back(snh / vol);
        out.ne.push_back(sne / vol);
        out.rk.push_back(srk / vol);
        if (sm > 0.0) {
            out.x1.push_back(smx1 / sm); out.x2.push_back(smx2 / sm); out.x3.push_back(smx3 / sm);
        } else if (sv > 0.0) {
            out.x1.push_back(svx1 / sv); out.x2.push_back(svx2 / sv); out.x3.push_back(svx3 / sv);
        } else {
            out.x1.push_back(1.0); out.x2.push_back(1.0); out.x3.push_back(0.0);
        }
        out.te.push_back(st > 0.0 ? ste / st : sv > 0.0 ? svte / sv : in.te_min);
    }
};

void integrals(long long n, const double* nH, const double* x1, const double* x2, const double* x3, const double* ne,
               const double* te, const double* rk, double yHe, const std::vector<double>& vol, double* a) {
    for (int q = 0; q < 7; ++q) a[q] = 0.0;
    for (long long i = 0; i < n; ++i) {
        const double v = vol[i];
        a[0] = a[0] + nH[i] * v;
        a[1] = a[1] + nH[i] * x1[i] * v;
        a[2] = a[2] + nH[i] * yHe * x2[i] * v;
        a[3] = a[3] + nH[i] * yHe * x3[i] * v;
        a[4] = a[4] + ne[i] * v;
        a[5] = a[5] + (rk ? rk[i] : 0.0) * v;
        a[6] = a[6] + (nH[i] * (1.0 + yHe) + ne[i]) * te[i] * v;
    }
}

}  // namespace

bool refine_plan(const OctHost& o, const RefineIn& in, RefineOut& out, std::string* err) {
    const int nold = o.nleaf;
    out = RefineOut();
    Planner p{o, in, std::vector<char>(nold, 0), out};
    for (int il = 0; il < nold; ++il) {   // front flags (:66-88)
        if (in.nH[il] <= 0.0) continue;
        const double xr = in.xHI[il];
        if (xr > in.eps && xr < 1.0 - in.eps) {
            p.front[il] = 1;
            continue;
        }
        const int c = o.cell_of_leaf[il];
        for (int f = 0; f < 6; ++f) {
            const int jc = o.nbr[8 * (size_t)c + f];
            if (jc < 0) continue;
            const int jl = o.ileaf[jc];
            if (jl < 0 || in.nH[jl] <= 0.0) continue;
            if (std::fabs(in.xHI[jl] - xr) > in.dx) {
                p.front[il] = 1;
                break;
            }
        }
    }
    for (char f : p.front) out.nfront += f;
    p.build(0.0, 0.0, 0.0, o.half, 0);
    const size_t nn = out.x.size();
    for (size_t i = 0; i < nn && !p.overflow; ++i) p.remap(out.x[i], out.y[i], out.z[i], o.half / std::ldexp(1.0, out.lev[i]));
    if (p.overflow) {
        if (err) *err = "re-refinement: octree descent stack overflow";
        return false;
    }
    std::vector<double> lh(nold);
    for (int il = 0; il < nold; ++il) lh[il] = o.lgeo[4 * (size_t)il + 3];
    return refine_check(in, lh, o.half, out, err);
}

// conservation_report (:299-352): the seven box integrals before (old leaf
// half widths lh) and after, the largest relative change at most 1e-8.
bool refine_check(const RefineIn& in, const std::vector<double>& lh, double half, RefineOut& out, std::string* err) {
    const long long nold = (long long)lh.size();
    const size_t nn = out.x.size();
    std::vector<double> vold(nold), vnew(nn);
    for (long long il = 0; il < nold; ++il) {
        const double w = 2.0 * lh[il];
        vold[il] = w * w * w;
    }
    for (size_t i = 0; i < nn; ++i) {
        const double w = 2.0 * half / std::ldexp(1.0, out.lev[i]);
        vnew[i] = w * w * w;
    }
    integrals(nold, in.nH, in.xHI, in.xHeI, in.xHeII, in.ne, in.Te, in.rk, in.yHe, vold, out.before);
    integrals((long long)nn, out.nH.data(), out.x1.data(), out.x2.data(), out.x3.data(), out.ne.data(), out.te.data(),
              in.rk ? out.rk.data() : nullptr, in.yHe, vnew, out.after);
    out.worst = 0.0;
    for (int q = 0; q < 7; ++q)
        if (std::fabs(out.before[q]) > 0.0)
            out.worst = std::max(out.worst, std::fabs(out.after[q] - out.before[q]) / std::fabs(out.before[q]));
    if (out.worst > 1.0e-8) {
        if (err) *err = "re-refinement lost " + std::to_string(out.worst) + " of a conserved box integral";
        return false;
    }
    return true;
}

// The generic text leaf list ("nleaf boxlen", then "x y z level nH") with the
// remapped x_HI, x_HeI, x_HeII, n_e, T_e and rhokap as extra columns (the
// reader takes the first five).
bool refine_write(const std::string& path, double boxlen, const RefineOut& r, std::string* err) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) {
        if (err) *err = "cannot write " + path;
        return false;
    }
    std::fprintf(f, "%zu %.17g\n", r.x.size(), boxlen);
    // std::to_chars in general format with precision 17 writes what printf's
    // %.17g does, without the format parsing
    std::vector<char> buf;
    buf.reserve(1 << 22);
    char tmp[64];
    auto put = [&](double v, char sep) {
        const auto res = std::to_chars(tmp, tmp + sizeof(tmp), v, std::chars_format::general, 17);
        buf.insert(buf.end(), tmp, res.ptr);
        buf.push_back(sep);
    };
    for (size_t i = 0; i < r.x.size(); ++i) {
        put(r.x[i], ' ');
        put(r.y[i], ' ');
        put(r.z[i], ' ');
        const auto res = std::to_chars(tmp, tmp + sizeof(tmp), r.lev[i]);
        buf.insert(buf.end(), tmp, res.ptr);
        buf.push_back(' ');
        put(r.nH[i], ' ');
        put(r.x1[i], ' ');
        put(r.x2[i], ' ');
        put(r.x3[i], ' ');
        put(r.ne[i], ' ');
        put(r.te[i], ' ');
        put(r.rk[i], '\n');
        if (buf.size() > (1u << 22) - 512) {
            std::fwrite(buf.data(), 1, buf.size(), f);
            buf.clear();
        }
    }
    if (!buf.empty()) std::fwrite(buf.data(), 1, buf.size(), f);
    if (std::fclose(f) != 0) {
        if (err) *err = "cannot write " + path;
        return false;
    }
    return true;
}

}  // namespace mochii

using namespace mochii;

namespace {
thread_local std::string g_refine_err;
}

extern "C" int mochii_refine_plan(const char* in_list, const double* nH, const double* xHI, const double* xHeI,
                                  const double* xHeII, const double* ne, const double* Te, const double* rhokap,
                                  double He_abund, double te_min, int lbase, int lmax, double eps, double dx,
                                  const char* out_list, int64_t* counts2, double* worst) {
    if (!in_list || !nH || !xHI || !xHeI || !xHeII || !ne || !Te || !out_list || lbase < 0 || lmax < lbase ||
        lmax > 20)
        return MOCHII_ERR_BAD_PARAM;
    std::vector<double> lx, ly, lz, lnH;
    std::vector<int> lev;
    double boxlen = 0.0;
    OctHost o;
    if (!leaf_list_read(in_list, lx, ly, lz, lev, lnH, &boxlen, &g_refine_err) ||
        !octree_build(lx, ly, lz, lev, 0.5 * boxlen, o, &g_refine_err))
        return MOCHII_ERR_TABLE;
    RefineIn in{nH, xHI, xHeI, xHeII, ne, Te, rhokap, He_abund, te_min, lbase, lmax, eps, dx};
    RefineOut r;
    if (!refine_plan(o, in, r, &g_refine_err)) return MOCHII_ERR_BAD_PARAM;
    if (!refine_write(out_list, boxlen, r, &g_refine_err)) return MOCHII_ERR_BAD_PARAM;
    if (counts2) {
        counts2[0] = (int64_t)r.x.size();
        counts2[1] = r.nfront;
    }
    if (worst) *worst = r.worst;
    return MOCHII_OK;
}

extern "C" const char* mochii_refine_last_error(void) { return g_refine_err.c_str(); }

extern "C" int mochii_refine_front(mochii_ctx* c, const char* out_list, mochii_ctx** out) {
    if (!c || !out) return MOCHII_ERR_BAD_PARAM;
    if (c->oct.ncells == 0 || c->par.grid_car) {
        c->last_error = "mochii_refine_front: needs an octree grid (grid_type = 'amr')";
        return MOCHII_ERR_UNSUPPORTED;
    }
    const mochii_params& p = c->par;
    if (p.refine_lbase < 0 || p.refine_lmax < p.refine_lbase || p.refine_lmax > 20) {
        c->last_error = "mochii_refine_front: need 0 <= par%refine_lbase <= par%refine_lmax <= 20";
        return MOCHII_ERR_BAD_PARAM;
    }
    // the old state on the host for the conserved integrals
    const long long n = c->grid.nleaf;
    std::vector<double> f[6];
    const char* names[6] = {"nH", "x_HI", "x_HeI", "x_HeII", "n_e", "T_e"};
    for (int k = 0; k < 6; ++k) {
        f[k].resize((size_t)n);
        if (int rc = mochii_get_field(c, names[k], f[k].data(), n)) return rc;
    }
    std::vector<double> rk;
    if (c->rhokap) {
        rk.resize((size_t)n);
        if (cudaMemcpy(rk.data(), c->rhokap, (size_t)n * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
            return MOCHII_ERR_CUDA;
    }
    RefineIn in{f[0].data(), f[1].data(), f[2].data(), f[3].data(), f[4].data(), f[5].data(),
                c->rhokap ? rk.data() : nullptr, p.He_abund, p.te_min, p.refine_lbase, p.refine_lmax,
                p.refine_eps, p.refine_dx};
    RefineOut r;
    std::string why;
    if (!refine_plan_device(c, in, r, &why) || !refine_check(in, c->lhalf, c->oct.half, r, &why)) {
        c->last_error = "mochii_refine_front: " + why;
        return MOCHII_ERR_BAD_PARAM;
    }
    const double boxlen = 2.0 * c->oct.half;
    if (out_list && out_list[0] && !refine_write(out_list, boxlen, r, &why)) {
        c->last_error = "mochii_refine_front: " + why;
        return MOCHII_ERR_BAD_PARAM;
    }
    // the new context from the refined leaves in memory, its state from the remap
    mochii_params q = p;
    std::snprintf(q.amr_file, sizeof(q.amr_file), "%s", out_list && out_list[0] ? out_list : "(refined in memory)");
    const LeafList ll{&r.x, &r.y, &r.z, &r.nH, &r.lev, boxlen};
    mochii_ctx* nc = nullptr;
    g_leaf_preload = &ll;
    int rc = mochii_init(&q, &nc);
    g_leaf_preload = nullptr;
    if (rc) {
        c->last_error = std::string("mochii_refine_front: ") + mochii_last_error(nullptr);
        return rc;
    }
    const long long nn = (long long)r.x.size();
    const std::vector<double>* cols[5] = {&r.x1, &r.x2, &r.x3, &r.ne, &r.te};
    const char* set[5] = {"x_HI", "x_HeI", "x_HeII", "n_e", "T_e"};
    bool ok = true;
    for (int k = 0; ok && k < 5; ++k) ok = mochii_set_field(nc, set[k], cols[k]->data(), nn) == MOCHII_OK;
    if (!ok || (rc = mochii_opacity_fill(nc))) {
        mochii_destroy(nc);
        c->last_error = "mochii_refine_front: cannot set the remapped state";
        return rc ? rc : MOCHII_ERR_BAD_PARAM;
    }
    *out = nc;
    return MOCHII_OK;
}
