// Oracle (test infrastructure only): octree_mod.f90 restatement.
#include "orc_amr.h"

#include <fstream>
#include <sstream>

#include "orc_core.h"

namespace orc {

void Octree::build(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z,
                   const std::vector<int>& lev, double half) {
    xmin = ymin = zmin = -half;
    xmax = ymax = zmax = half;
    L = 2.0 * half;
    nleaf = (int)x.size();
    parent.assign(1, -1);
    level.assign(1, 0);
    ileaf.assign(1, -1);
    children.assign(8, -1);
    cx.assign(1, (xmin + xmax) * 0.5);
    cy.assign(1, (ymin + ymax) * 0.5);
    cz.assign(1, (zmin + zmax) * 0.5);
    ch.assign(1, L * 0.5);
    icell_of_leaf.assign(nleaf, -1);
    for (int il = 0; il < nleaf; ++il) {
        int icell = 0;
        for (int l = 0; l < lev[il]; ++l) {
            int ioct = 0;
            if (x[il] >= cx[icell]) ioct += 1;
            if (y[il] >= cy[icell]) ioct += 2;
            if (z[il] >= cz[icell]) ioct += 4;
            if (children[8 * icell + ioct] < 0) {
                const int nc = (int)parent.size();
                parent.push_back(icell);
                level.push_back(l + 1);
                ileaf.push_back(-1);
                for (int k = 0; k < 8; ++k) children.push_back(-1);
                const double h = ch[icell] * 0.5;
                ch.push_back(h);
                const int ix = ioct % 2, iy = (ioct / 2) % 2, iz = ioct / 4;
                cx.push_back(cx[icell] + (double)(2 * ix - 1) * h);
                cy.push_back(cy[icell] + (double)(2 * iy - 1) * h);
                cz.push_back(cz[icell] + (double)(2 * iz - 1) * h);
                children[8 * icell + ioct] = nc;
            }
            icell = children[8 * icell + ioct];
        }
        ileaf[icell] = il;
        icell_of_leaf[il] = icell;
    }
    ncells = (int)parent.size();
    build_neighbors();
}

int Octree::find_cell_at_level(double x, double y, double z, int target) const {
    if (x < xmin || x > xmax || y < ymin || y > ymax || z < zmin || z > zmax) return -1;
    int icell = 0;
    for (;;) {
        if (level[icell] >= target) return icell;
        if (ileaf[icell] >= 0) return icell;
        int ioct = 0;
        if (x >= cx[icell]) ioct += 1;
        if (y >= cy[icell]) ioct += 2;
        if (z >= cz[icell]) ioct += 4;
        const int c = children[8 * icell + ioct];
        if (c < 0) return icell;
        icell = c;
    }
}

void Octree::build_neighbors() {
    neighbor.assign((size_t)6 * ncells, -1);
    for (int icell = 0; icell < ncells; ++icell) {
        const double x = cx[icell], y = cy[icell], z = cz[icell], hp = 2.0 * ch[icell];
        const int lv = level[icell];
        int* nb = &neighbor[6 * (size_t)icell];
        if (x + hp <= xmax) nb[0] = find_cell_at_level(x + hp, y, z, lv);
        if (x - hp >= xmin) nb[1] = find_cell_at_level(x - hp, y, z, lv);
        if (y + hp <= ymax) nb[2] = find_cell_at_level(x, y + hp, z, lv);
        if (y - hp >= ymin) nb[3] = find_cell_at_level(x, y - hp, z, lv);
        if (z + hp <= zmax) nb[4] = find_cell_at_level(x, y, z + hp, lv);
        if (z - hp >= zmin) nb[5] = find_cell_at_level(x, y, z - hp, lv);
        for (int f = 0; f < 6; ++f) {   // a neighbour that is an ancestor is no neighbour
            const int n = nb[f];
            if (n < 0 || n == icell) continue;
            for (int c = parent[icell]; c >= 0; c = parent[c])
                if (c == n) {
                    nb[f] = -1;
                    break;
                }
        }
    }
}

int Octree::find_leaf(double x, double y, double z) const {
    if (x < xmin || x > xmax || y < ymin || y > ymax || z < zmin || z > zmax) return -1;
    int icell = 0;
    for (;;) {
        if (ileaf[icell] >= 0) return ileaf[icell];
        int ioct = 0;
        if (x >= cx[icell]) ioct += 1;
        if (y >= cy[icell]) ioct += 2;
        if (z >= cz[icell]) ioct += 4;
        icell = children[8 * icell + ioct];
        if (icell < 0) return -1;
    }
}

void Octree::cell_exit(int icell, double x, double y, double z, double kx, double ky, double kz, double* tout,
                       int* iface) const {
    const double h = ch[icell], ccx = cx[icell], ccy = cy[icell], ccz = cz[icell];
    double t[6];
    if (kx > 0.0) { t[0] = (ccx + h - x) / kx; t[1] = HUGEST; }
    else if (kx < 0.0) { t[0] = HUGEST; t[1] = (ccx - h - x) / kx; }
    else { t[0] = HUGEST; t[1] = HUGEST; }
    if (ky > 0.0) { t[2] = (ccy + h - y) / ky; t[3] = HUGEST; }
    else if (ky < 0.0) { t[2] = HUGEST; t[3] = (ccy - h - y) / ky; }
    else { t[2] = HUGEST; t[3] = HUGEST; }
    if (kz > 0.0) { t[4] = (ccz + h - z) / kz; t[5] = HUGEST; }
    else if (kz < 0.0) { t[4] = HUGEST; t[5] = (ccz - h - z) / kz; }
    else { t[4] = HUGEST; t[5] = HUGEST; }
    int f = 0;   // minloc: first minimum
    for (int k = 1; k < 6; ++k)
        if (t[k] < t[f]) f = k;
    *iface = f;
    *tout = t[f];
}

int Octree::next_leaf(int icell, int iface, double x, double y, double z) const {
    int n = neighbor[6 * (size_t)icell + iface];
    if (n < 0) return -1;
    while (ileaf[n] < 0) {
        int ioct = 0;
        switch (iface) {   // the face-normal octant bit is set by the face crossed
            case 0: if (y >= cy[n]) ioct += 2; if (z >= cz[n]) ioct += 4; break;
            case 1: ioct += 1; if (y >= cy[n]) ioct += 2; if (z >= cz[n]) ioct += 4; break;
            case 2: if (x >= cx[n]) ioct += 1; if (z >= cz[n]) ioct += 4; break;
            case 3: if (x >= cx[n]) ioct += 1; ioct += 2; if (z >= cz[n]) ioct += 4; break;
            case 4: if (x >= cx[n]) ioct += 1; if (y >= cy[n]) ioct += 2; break;
            default: if (x >= cx[n]) ioct += 1; if (y >= cy[n]) ioct += 2; ioct += 4; break;
        }
        const int c = children[8 * n + ioct];
        if (c < 0) break;
        n = c;
    }
    return ileaf[n];
}

bool read_leaf_list(const std::string& path, std::vector<double>& x, std::vector<double>& y,
                    std::vector<double>& z, std::vector<int>& lev, std::vector<double>& nH, double* boxlen,
                    std::string* err) {
    std::ifstream f(path);
    if (!f) {
        if (err) *err = "cannot open amr_file " + path;
        return false;
    }
    long long n = 0;
    double bl = 0.0;
    std::string line;
    if (!std::getline(f, line) || !(std::istringstream(line) >> n >> bl) || n < 1) {
        if (err) *err = "bad amr_file header";
        return false;
    }
    x.resize(n); y.resize(n); z.resize(n); lev.resize(n); nH.resize(n);
    for (long long i = 0; i < n; ++i) {
        if (!std::getline(f, line)) {
            if (err) *err = "amr_file ends early";
            return false;
        }
        std::istringstream s(line);
        if (!(s >> x[i] >> y[i] >> z[i] >> lev[i] >> nH[i])) {
            if (err) *err = "bad amr_file row";
            return false;
        }
    }
    *boxlen = bl;
    return true;
}

// ---- amr_refine_mod.f90 ----------------------------------------------------
namespace {

struct Refiner {
    const Octree& o;
    const std::vector<double>* st;   // nH, xHI, xHeI, xHeII, ne, Te
    const std::vector<double>& rk;
    double yHe, te_min;
    int lbase, lmax;
    std::vector<char> front;
    RefineResult& r;
    bool overflow = false;

    bool cell_has_front(double x, double y, double z, double h) {   // :398-422
        std::vector<int> stk{0};
        while (!stk.empty()) {
            const int ic = stk.back();
            stk.pop_back();
            if (std::fabs(o.cx[ic] - x) > o.ch[ic] + h) continue;
            if (std::fabs(o.cy[ic] - y) > o.ch[ic] + h) continue;
            if (std::fabs(o.cz[ic] - z) > o.ch[ic] + h) continue;
            if (o.ileaf[ic] >= 0) {
                if (front[o.ileaf[ic]]) return true;
                continue;
            }
            for (int k = 0; k < 8; ++k)
                if (o.children[8 * ic + k] >= 0) {
                    if (stk.size() >= 512) { overflow = true; return false; }
                    stk.push_back(o.children[8 * ic + k]);
                }
        }
        return false;
    }

    void rec_build(double x, double y, double z, double h, int level) {   // :355-380
        if ((level < lmax && cell_has_front(x, y, z, h)) || level < lbase) {
            const double hc = 0.5 * h;
            for (int iz = 0; iz <= 1; ++iz)
                for (int iy = 0; iy <= 1; ++iy)
                    for (int ix = 0; ix <= 1; ++ix)
                        rec_build(x + (double)(2 * ix - 1) * hc, y + (double)(2 * iy - 1) * hc,
                                  z + (double)(2 * iz - 1) * hc, hc, level + 1);
        } else {
            r.x.push_back(x); r.y.push_back(y); r.z.push_back(z); r.lev.push_back(level);
        }
    }

    static double ov1(double ca, double ha, double cb, double hb) {   // overlap_1d, :186-190
        const double v = std::min(ca + ha, cb + hb) - std::max(ca - ha, cb - hb);
        return v < 0.0 ? 0.0 : v;
    }

    void remap_leaf(double x, double y, double z, double h) {   // :197-292
        const std::vector<double> &nH = st[0], &xHI = st[1], &xHeI = st[2], &xHeII = st[3], &ne = st[4], &Te = st[5];
        double sv = 0, snh = 0, sne = 0, srk = 0, sm = 0, smx1 = 0, smx2 = 0, smx3 = 0, ssum = 0, ste = 0;
        double svx1 = 0, svx2 = 0, svx3 = 0, svte = 0;
        std::vector<int> stk{0};
        while (!stk.empty()) {
            const int ic = stk.back();
            stk.pop_back();
            const double hw = o.ch[ic];
            if (std::fabs(o.cx[ic] - x) >= hw + h) continue;
            if (std::fabs(o.cy[ic] - y) >= hw + h) continue;
            if (std::fabs(o.cz[ic] - z) >= hw + h) continue;
            if (o.ileaf[ic] >= 0) {
                const int jl = o.ileaf[ic];
                const double ov = ov1(o.cx[ic], hw, x, h) * ov1(o.cy[ic], hw, y, h) * ov1(o.cz[ic], hw, z, h);
                if (ov <= 0.0) continue;
                sv = sv + ov;
                snh = snh + nH[jl] * ov;
                sne = sne + ne[jl] * ov;
                srk = srk + (rk.empty() ? 0.0 : rk[jl]) * ov;
                const double wm = nH[jl] * ov;
                sm = sm + wm;
                smx1 = smx1 + wm * xHI[jl];
                smx2 = smx2 + wm * xHeI[jl];
                smx3 = smx3 + wm * xHeII[jl];
                const double wt = (nH[jl] * (1.0 + yHe) + ne[jl]) * ov;
                ssum = ssum + wt;
                ste = ste + wt * Te[jl];
                svx1 = svx1 + ov * xHI[jl];
                svx2 = svx2 + ov * xHeI[jl];
                svx3 = svx3 + ov * xHeII[jl];
                svte = svte + ov * Te[jl];
                continue;
            }
            for (int k = 0; k < 8; ++k)
                if (o.children[8 * ic + k] >= 0) {
                    if (stk.size() >= 512) { overflow = true; return; }
                    stk.push_back(o.children[8 * ic + k]);
                }
        }
        const double vol = (2.0 * h) * (2.0 * h) * (2.0 * h);
        r.nH.push_back(snh / vol);
        r.ne.push_back(sne / vol);
        r.rk.push_back(srk / vol);
        if (sm > 0.0) { r.x1.push_back(smx1 / sm); r.x2.push_back(smx2 / sm); r.x3.push_back(smx3 / sm); }
        else if (sv > 0.0) { r.x1.push_back(svx1 / sv); r.x2.push_back(svx2 / sv); r.x3.push_back(svx3 / sv); }
        else { r.x1.push_back(1.0); r.x2.push_back(1.0); r.x3.push_back(0.0); }
        r.te.push_back(ssum > 0.0 ? ste / ssum : sv > 0.0 ? svte / sv : te_min);
    }
};

}  // namespace

bool refine_front(const Octree& o, const std::vector<double>* st6, const std::vector<double>& rk, double yHe,
                  double te_min, int lbase, int lmax, double eps, double dx, RefineResult& r, std::string* err) {
    r = RefineResult();
    Refiner R{o, st6, rk, yHe, te_min, lbase, lmax, std::vector<char>(o.nleaf, 0), r};
    const std::vector<double> &nH = st6[0], &xHI = st6[1];
    for (int il = 0; il < o.nleaf; ++il) {   // :66-88
        if (nH[il] <= 0.0) continue;
        const double xr = xHI[il];
        if (xr > eps && xr < 1.0 - eps) { R.front[il] = 1; continue; }
        const int ic = o.icell_of_leaf[il];
        for (int f = 0; f < 6; ++f) {
            const int jc = o.neighbor[6 * ic + f];
            if (jc < 0) continue;
            const int jl = o.ileaf[jc];
            if (jl < 0 || nH[jl] <= 0.0) continue;
            if (std::fabs(xHI[jl] - xr) > dx) { R.front[il] = 1; break; }
        }
    }
    for (char f : R.front) r.nfront += f;
    const double half = 0.5 * o.L;
    R.rec_build(0.0, 0.0, 0.0, half, 0);
    for (size_t i = 0; i < r.x.size() && !R.overflow; ++i)
        R.remap_leaf(r.x[i], r.y[i], r.z[i], half / std::pow(2.0, r.lev[i]));
    if (R.overflow) { if (err) *err = "descent stack overflow"; return false; }
    // conservation_report, :299-352
    double a[7] = {}, b[7] = {};
    for (int il = 0; il < o.nleaf; ++il) {
        const double w = 2.0 * o.ch[o.icell_of_leaf[il]], v = w * w * w;
        a[0] += st6[0][il] * v;
        a[1] += st6[0][il] * st6[1][il] * v;
        a[2] += st6[0][il] * yHe * st6[2][il] * v;
        a[3] += st6[0][il] * yHe * st6[3][il] * v;
        a[4] += st6[4][il] * v;
        a[5] += (rk.empty() ? 0.0 : rk[il]) * v;
        a[6] += (st6[0][il] * (1.0 + yHe) + st6[4][il]) * st6[5][il] * v;
    }
    for (size_t i = 0; i < r.x.size(); ++i) {
        const double w = 2.0 * half / std::pow(2.0, r.lev[i]), v = w * w * w;
        b[0] += r.nH[i] * v;
        b[1] += r.nH[i] * r.x1[i] * v;
        b[2] += r.nH[i] * yHe * r.x2[i] * v;
        b[3] += r.nH[i] * yHe * r.x3[i] * v;
        b[4] += r.ne[i] * v;
        b[5] += (rk.empty() ? 0.0 : r.rk[i]) * v;
        b[6] += (r.nH[i] * (1.0 + yHe) + r.ne[i]) * r.te[i] * v;
    }
    for (int q = 0; q < 7; ++q)
        if (std::fabs(a[q]) > 0.0) r.worst = std::max(r.worst, std::fabs(b[q] - a[q]) / std::fabs(a[q]));
    if (r.worst > 1.0e-8) { if (err) *err = "a conserved box integral moved"; return false; }
    return true;
}

}  // namespace orc
