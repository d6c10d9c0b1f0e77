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

}  // namespace orc
