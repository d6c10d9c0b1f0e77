// AMR octree (octree_mod.f90): host build from a leaf list and the device
// layout the walk kernels read.
//
// Cells are renumbered breadth first (level-major) after the build, so the
// complete top levels are one contiguous block that the launch kernel stages
// in shared memory for the leaf search (up to levels 0..3, 585 cells).  The walk
// is leaf-indexed: per leaf one 32-byte record (centre, half width) and one
// 32-byte row of what lies across each face -- the neighbouring leaf when
// the face neighbour is a leaf (the common case), else the internal cell to
// descend from (encoded -2 - cell), -1 outside the box.  Cell tables
// (geometry, children, leaf of cell) are read only for those descents and
// the leaf search at launch.  Leaves keep the file order (the generator
// writes them in Morton order, i.e. depth-first, so spatial neighbours are
// neighbours in memory).
#pragma once
#include <vector_types.h>

#include <string>
#include <vector>

namespace mochii {

constexpr int kOctShared = 585;   // levels 0..3 of a complete tree

struct OctHost {
    int ncells = 0, nleaf = 0, nshared = 0;   // cells 0..nshared-1: complete top levels
    double half = 0.0;                            // box half width (box centred on 0)
    std::vector<double> geo;                      // 4 per cell: cx, cy, cz, ch
    std::vector<int> children;                    // 8 per cell, -1 none
    std::vector<int> nbr;                         // 8 per cell (6 faces + 2 pad), -1 outside
    std::vector<int> ileaf;                       // per cell, -1 internal
    std::vector<int> cell_of_leaf;                // per leaf
    std::vector<int> level;                       // per cell
    std::vector<double> lgeo;                     // 4 per leaf: cx, cy, cz, half width
    std::vector<int> lnext;                       // 8 per leaf (6 faces + 2 pad)
};

// The device copy (pointers into one allocation).
struct OctDev {
    int ncells = 0;            // 0: Cartesian grid
    int nshared = 0;           // cells 0..nshared-1 are the complete top levels (staged)
    double half = 0.0;
    const double4* geo = nullptr;       // per cell
    const int* children = nullptr;      // 8 per cell
    const int* ileaf = nullptr;         // per cell
    const double4* lgeo = nullptr;      // per leaf
    const int* lnext = nullptr;         // 8 per leaf
    // the car grid walked as an octree (par%car_walk = 'amr'): leaves in
    // raster order, no cell tables; the start leaf is car_index
    int car = 0;
    int n[3] = {0, 0, 0};
    double org[3] = {0.0, 0.0, 0.0};   // xmin, ymin, zmin
    double hi[3] = {0.0, 0.0, 0.0};    // xmax, ymax, zmax
    double dcell = 0.0;
};

// read_generic_amr.f90:60-81 text leaf list: "nleaf boxlen", then
// "x y z level nH [...]" per leaf, coordinates centred on the box.
bool leaf_list_read(const std::string& path, std::vector<double>& x, std::vector<double>& y, std::vector<double>& z,
                    std::vector<int>& lev, std::vector<double>& nH, double* boxlen, std::string* err);
// amr_build_tree + amr_build_neighbors (octree_mod.f90:342-479).
bool octree_build(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z,
                  const std::vector<int>& lev, double half, OctHost& o, std::string* err);
// The walk tables of the namelist car grid for par%car_walk = 'amr':
// cell_cx/cy/cz/ch (octree_mod.f90:113-153) and car_next (:620-641).
void car_walk_tables(int nx, int ny, int nz, double xmin, double ymin, double zmin, double dcell, OctHost& o);

// A leaf list held in memory: set by the re-refinement around the
// mochii_init of the refined context, which then takes its leaves from here
// instead of reading par%amr_file (same thread only).
struct LeafList {
    const std::vector<double>*x, *y, *z, *nH;
    const std::vector<int>* lev;
    double boxlen;
};
extern thread_local const LeafList* g_leaf_preload;

}  // namespace mochii
