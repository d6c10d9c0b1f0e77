// Solution-driven I-front re-refinement (amr_refine_mod.f90): the plan's
// inputs and outputs, shared by the host plan (refine.cpp) and the device
// plan (refine_dev.cu).
#pragma once
#include <string>
#include <vector>

struct mochii_ctx;

namespace mochii {

struct RefineIn {
    const double *nH, *xHI, *xHeI, *xHeII, *ne, *Te, *rk;   // rk may be null (no grains)
    double yHe, te_min;
    int lbase, lmax;
    double eps, dx;
};

// The new leaves in depth-first order (octants ix + 2 iy + 4 iz) with the
// remapped state, the front count and the conserved integrals.
struct RefineOut {
    std::vector<double> x, y, z, nH, x1, x2, x3, ne, te, rk;
    std::vector<int> lev;
    long long nfront = 0;
    double before[7] = {}, after[7] = {}, worst = 0.0;
};

// conservation_report (amr_refine_mod.f90:299-352): out's seven box
// integrals before (the old state in in, old leaf half widths lh) and after,
// and their largest relative change, which must stay within 1e-8.
bool refine_check(const RefineIn& in, const std::vector<double>& lh, double half, RefineOut& out, std::string* err);

// The device plan for a context on an octree: the front flags from its
// device state and leaf neighbours, the new tree built level by level (one
// thread per cell of a level, the cells that hold a front leaf split, the
// leaves sorted into depth-first order by their octant path), the remap one
// thread per new leaf.  Fills out's leaves, state and nfront (the integrals
// are the caller's); in.* are ignored except the levels and thresholds.
bool refine_plan_device(mochii_ctx* c, const RefineIn& in, RefineOut& out, std::string* err);

}  // namespace mochii
