// Host build of the AMR octree: insertion of the leaves (octree_mod.f90:342-432),
// breadth-first renumbering, and the face-neighbour table (:447-479).
#include <cuda_runtime.h>

#include <algorithm>
#include <fstream>
#include <sstream>

#include "octree.h"

namespace mochii {

bool leaf_list_read(const std::string& path, std::vector<double>& x, std::vector<double>& y, std::vector<double>& z,
                    std::vector<int>& lev, std::vector<double>& nH, double* boxlen, std::string* err) {
    std::ifstream f(path);
    if (!f) {
        if (err) *err = "cannot open par%amr_file " + path;
        return false;
    }
    std::string line;
    long long n = 0;
    double bl = 0.0;
    if (!std::getline(f, line) || !(std::istringstream(line) >> n >> bl) || n < 1 || !(bl > 0.0)) {
        if (err) *err = path + ": header must be 'nleaf boxlen'";
        return false;
    }
    x.resize(n); y.resize(n); z.resize(n); lev.resize(n); nH.resize(n);
    for (long long i = 0; i < n; ++i) {
        if (!std::getline(f, line)) {
            if (err) *err = path + ": fewer leaf rows than the header states";
            return false;
        }
        std::istringstream s(line);
        if (!(s >> x[i] >> y[i] >> z[i] >> lev[i] >> nH[i]) || lev[i] < 0 || lev[i] > 20) {
            if (err) *err = path + ": bad leaf row " + std::to_string(i + 1);
            return false;
        }
    }
    *boxlen = bl;
    return true;
}

bool octree_build(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z,
                  const std::vector<int>& lev, double half, OctHost& o, std::string* err) {
    const int nleaf = (int)x.size();
    // insertion in leaf order (build numbering)
    std::vector<int> parent{-1}, level{0}, ileaf{-1}, children(8, -1), col(nleaf, -1);
    std::vector<double> cx{0.0}, cy{0.0}, cz{0.0}, ch{half};
    for (int il = 0; il < nleaf; ++il) {
        int icell = 0;
        for (int l = 0; l < lev[il]; ++l) {
            int ioct = 0;
            if (x[il] >= cx[icell]) ioct += 1;
            if (y[il] >= cy[icell]) ioct += 2;
            if (z[il] >= cz[icell]) ioct += 4;
            if (ileaf[icell] >= 0) {
                if (err) *err = "par%amr_file: leaf " + std::to_string(il + 1) + " lies inside another leaf";
                return false;
            }
            if (children[8 * icell + ioct] < 0) {
                const int nc = (int)parent.size();
                parent.push_back(icell);
                level.push_back(l + 1);
                ileaf.push_back(-1);
                children.insert(children.end(), 8, -1);
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
        if (ileaf[icell] >= 0 || children[8 * icell] >= 0 || children[8 * icell + 7] >= 0) {
            if (err) *err = "par%amr_file: leaf " + std::to_string(il + 1) + " repeats or encloses another leaf";
            return false;
        }
        ileaf[icell] = il;
        col[il] = icell;
    }
    const int nc = (int)parent.size();
    // breadth-first renumbering: stable by level, then by build order
    std::vector<int> order(nc), newid(nc);
    for (int i = 0; i < nc; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return level[a] < level[b]; });
    for (int i = 0; i < nc; ++i) newid[order[i]] = i;
    o = OctHost();
    o.ncells = nc;
    o.nleaf = nleaf;
    o.half = half;
    o.geo.resize(4 * (size_t)nc);
    o.children.assign(8 * (size_t)nc, -1);
    o.ileaf.resize(nc);
    o.level.resize(nc);
    std::vector<int> par_new(nc);
    for (int i = 0; i < nc; ++i) {
        const int old = order[i];
        o.geo[4 * i + 0] = cx[old];
        o.geo[4 * i + 1] = cy[old];
        o.geo[4 * i + 2] = cz[old];
        o.geo[4 * i + 3] = ch[old];
        for (int k = 0; k < 8; ++k) {
            const int c = children[8 * old + k];
            o.children[8 * i + k] = c < 0 ? -1 : newid[c];
        }
        o.ileaf[i] = ileaf[old];
        o.level[i] = level[old];
        par_new[i] = parent[old] < 0 ? -1 : newid[parent[old]];
    }
    o.cell_of_leaf.resize(nleaf);
    for (int il = 0; il < nleaf; ++il) o.cell_of_leaf[il] = newid[col[il]];
    // amr_find_cell_at_level (octree_mod.f90:679-698)
    auto at_level = [&](double px, double py, double pz, int target) {
        if (px < -half || px > half || py < -half || py > half || pz < -half || pz > half) return -1;
        int c = 0;
        for (;;) {
            if (o.level[c] >= target || o.ileaf[c] >= 0) return c;
            int ioct = 0;
            if (px >= o.geo[4 * c + 0]) ioct += 1;
            if (py >= o.geo[4 * c + 1]) ioct += 2;
            if (pz >= o.geo[4 * c + 2]) ioct += 4;
            const int ch2 = o.children[8 * c + ioct];
            if (ch2 < 0) return c;
            c = ch2;
        }
    };
    o.nbr.assign(8 * (size_t)nc, -1);
    for (int c = 0; c < nc; ++c) {
        const double px = o.geo[4 * c], py = o.geo[4 * c + 1], pz = o.geo[4 * c + 2], hp = 2.0 * o.geo[4 * c + 3];
        const int lv = o.level[c];
        int* nb = &o.nbr[8 * (size_t)c];
        if (px + hp <= half) nb[0] = at_level(px + hp, py, pz, lv);
        if (px - hp >= -half) nb[1] = at_level(px - hp, py, pz, lv);
        if (py + hp <= half) nb[2] = at_level(px, py + hp, pz, lv);
        if (py - hp >= -half) nb[3] = at_level(px, py - hp, pz, lv);
        if (pz + hp <= half) nb[4] = at_level(px, py, pz + hp, lv);
        if (pz - hp >= -half) nb[5] = at_level(px, py, pz - hp, lv);
        for (int f = 0; f < 6; ++f) {   // an ancestor is not a neighbour
            if (nb[f] < 0 || nb[f] == c) continue;
            for (int a = par_new[c]; a >= 0; a = par_new[a])
                if (a == nb[f]) {
                    nb[f] = -1;
                    break;
                }
        }
    }
    // the complete top levels of internal cells, at most kOctShared cells
    int ns = o.ileaf[0] < 0 ? 1 : 0;
    for (int lv = 0; ns > 0; ++lv) {
        const int next = ns + (1 << (3 * (lv + 1)));
        if (next > kOctShared || next > nc) break;
        bool complete = true;
        for (int c = ns; c < next && complete; ++c) complete = o.level[c] == lv + 1 && o.ileaf[c] < 0;
        if (!complete) break;
        ns = next;
    }
    o.nshared = ns;
    // leaf-indexed walk tables
    o.lgeo.resize(4 * (size_t)nleaf);
    o.lnext.assign(8 * (size_t)nleaf, -1);
    for (int il = 0; il < nleaf; ++il) {
        const int c = o.cell_of_leaf[il];
        for (int k = 0; k < 4; ++k) o.lgeo[4 * (size_t)il + k] = o.geo[4 * (size_t)c + k];
        for (int f = 0; f < 6; ++f) {
            const int nb = o.nbr[8 * (size_t)c + f];
            o.lnext[8 * (size_t)il + f] = nb < 0 ? -1 : o.ileaf[nb] >= 0 ? o.ileaf[nb] : -2 - nb;
        }
    }
    return true;
}

void car_walk_tables(int nx, int ny, int nz, double xmin, double ymin, double zmin, double dcell, OctHost& o) {
    o = OctHost();
    const long long n = (long long)nx * ny * nz;
    o.nleaf = (int)n;
    o.half = 0.5 * (dcell * nx);
    o.lgeo.resize(4 * (size_t)n);
    o.lnext.assign(8 * (size_t)n, -1);
    long long il = 0;
    for (int iz = 0; iz < nz; ++iz)
        for (int iy = 0; iy < ny; ++iy)
            for (int ix = 0; ix < nx; ++ix, ++il) {
                double* g = &o.lgeo[4 * (size_t)il];
                g[0] = xmin + ((double)ix + 0.5) * dcell;
                g[1] = ymin + ((double)iy + 0.5) * dcell;
                g[2] = zmin + ((double)iz + 0.5) * dcell;
                g[3] = 0.5 * dcell;
                int* f = &o.lnext[8 * (size_t)il];
                if (ix + 1 < nx) f[0] = (int)(il + 1);
                if (ix > 0) f[1] = (int)(il - 1);
                if (iy + 1 < ny) f[2] = (int)(il + nx);
                if (iy > 0) f[3] = (int)(il - nx);
                if (iz + 1 < nz) f[4] = (int)(il + (long long)nx * ny);
                if (iz > 0) f[5] = (int)(il - (long long)nx * ny);
            }
}

thread_local const LeafList* g_leaf_preload = nullptr;

}  // namespace mochii
