// Oracle (test infrastructure only): the AMR octree of octree_mod.f90 --
// tree build from a leaf list, face-neighbour table, leaf finder, cell exit
// and the neighbour step -- and the generic text leaf-list reader
// (read_generic_amr.f90).
#pragma once
#include <string>
#include <vector>

namespace orc {

struct Octree {                          // octree_mod.f90:20-61 (0-based indices, -1 = none)
    double xmin, xmax, ymin, ymax, zmin, zmax, L;
    int ncells = 0, nleaf = 0;
    std::vector<int> parent, level, ileaf, icell_of_leaf;
    std::vector<int> children;           // 8 per cell
    std::vector<int> neighbor;           // 6 per cell, -1 outside
    std::vector<double> cx, cy, cz, ch;
    void build(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z,
               const std::vector<int>& lev, double half);                      // :342-432
    void build_neighbors();                                                     // :447-479
    int find_leaf(double x, double y, double z) const;                         // :69-93
    int find_cell_at_level(double x, double y, double z, int target) const;    // :679-698
    void cell_exit(int icell, double x, double y, double z, double kx, double ky, double kz, double* t,
                   int* iface) const;                                           // :308-340
    int next_leaf(int icell, int iface, double x, double y, double z) const;   // :499-537
};

// Generic text leaf list (read_generic_amr.f90:60-81): "nleaf boxlen", then
// "x y z level nH [...]" per leaf, coordinates centred on the box.
bool read_leaf_list(const std::string& path, std::vector<double>& x, std::vector<double>& y,
                    std::vector<double>& z, std::vector<int>& lev, std::vector<double>& nH, double* boxlen,
                    std::string* err);

// amr_refine_front (amr_refine_mod.f90:46-436): front flags on the old
// leaves, the new leaf list (rec_build / cell_has_front), the overlap-volume
// remap (remap_leaf) and the conserved box integrals (conservation_report).
// st6 = nH, x_HI, x_HeI, x_HeII, n_e, T_e per old leaf; rk may be empty.
struct RefineResult {
    std::vector<double> x, y, z, nH, x1, x2, x3, ne, te, rk;
    std::vector<int> lev;
    long long nfront = 0;
    double worst = 0.0;
};
bool refine_front(const Octree& o, const std::vector<double>* st6, const std::vector<double>& rk, double yHe,
                  double te_min, int lbase, int lmax, double eps, double dx, RefineResult& r, std::string* err);

}  // namespace orc
