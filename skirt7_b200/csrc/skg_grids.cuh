// skg_grids.cuh -- device views of the dust grids and their path steppers.
//
// A stepper produces the segments (cell m, length ds) of DustGrid::path one at a time, in the
// order DustGridPath::addSegment receives them, without materialising the segment list.  The
// FP64 instantiation repeats the reference's arithmetic operation for operation (compile its
// users with --fmad=false for bit-identical cell sequences); the FP32 instantiation is the
// production geometry.
//   Cartesian : CartesianDustGrid::path   (SKIRTcore/CartesianDustGrid.cpp:136-283)
//   Tree      : TreeDustGrid::path        (SKIRTcore/TreeDustGrid.cpp:371-643)
//   Voronoi   : VoronoiMesh::path         (SKIRTcore/VoronoiMesh.cpp:778-873)
#pragma once
#include "skg_device.cuh"
#include <type_traits>
#include "../../include/skirt_b200.h"

namespace skg {

// Device view of a grid.  Both precisions are resident; kernels pick one by template.
struct DevGrid {
    int type;
    double xmin, ymin, zmin, xmax, ymax, zmax;
    double eps;                 // 1e-12 |diag| (TreeDustGrid.cpp:74, VoronoiMesh.cpp:220)
    float  epsf;                // FP32 nudge (a few ulps of the domain size)
    int ncells;
    int max_steps;

    // Cartesian planes
    int nx, ny, nz;
    const double *xv, *yv, *zv;
    const float  *xvf, *yvf, *zvf;
    // evenly spaced planes on every axis (plane q at corg + q * cstep): the FP32 walk computes its
    // walls instead of loading them
    int cart_uniform;
    float corg[3], cstep[3];

    // tree: node_box (6 doubles per node); nodef: 2 float4 per node
    //   nodef[2l]   = (xmin, ymin, zmin, int child0 or -1)
    //   nodef[2l+1] = (xmax, ymax, zmax, int cell or -1)
    int nnodes;
    const double* node_box;
    const int*    node_child;
    const int*    node_father;
    const int*    node_cell;
    const signed char* node_dir;
    const float4* nodef;
    const int*    nbroff;       // 6*nnodes+1
    const int*    nbr;
    const int*    cell_node;    // leaf node of each cell (TreeDustGrid::_idv)
    int search;
    // FP32 walk on the rope-linked tree (build_rope_tree): 64-byte leaf records in depth-first
    // order holding box, density, cell number and one rope per wall; 48-byte internal records
    // holding the split point and the child references
    const float4* lrec;
    const float4* irec;
    const int*    cell_leaf;    // cell number -> leaf index
    int root_ref;
    // lattice form (trees split at midpoints): 32-byte leaf records in cell order, walls at
    // fmaf(integer, lunit, lorg); irec as above (layout: RopeTree in skg_tree.h)
    const uint4*  prec;
    int lattice;
    float lorg[3], lunit[3];

    // Voronoi: sites (3 doubles / float4), CSR neighbours, FP32 bisector planes per CSR entry
    // vplane[q] = (n.x, n.y, n.z, n.p) with n = p_i - p_r and p the bisector midpoint; walls are
    // encoded as axis planes, so s = (n.p - n.r)/(n.k) for every entry with n.k > 0.
    int nsites;
    const double* site;
    const float4* sitef;
    const int*    vnoff;
    const int*    vnbr;
    const float4* vplane;
    const int4*   vnext;       // per CSR entry: (neighbour, its first entry, its end entry, 0)
    int nb;
    const int*    boff;
    const int*    bids;
    const double* vbbox;
    const double* vvol;        // Voronoi cell volumes
};

// The FP32 walk a grid takes.  Trees: the node walk (Bookkeeping search), the 64-byte rope records
// or their lattice form; Cartesian grids: the plane tables, or computed walls when every axis is
// evenly spaced.
enum TreeWalk : int { TW_ROPE = 0, TW_NODES = 1, TW_LATTICE = 2 };
enum CartWalk : int { CW_TABLE = 0, CW_UNIFORM = 1 };
inline int tree_walk_of(const DevGrid& g) {
    if (g.type == SKG_GRID_CARTESIAN) return g.cart_uniform ? CW_UNIFORM : CW_TABLE;
    return g.search == SKG_SEARCH_BOOKKEEPING ? TW_NODES : g.lattice ? TW_LATTICE : TW_ROPE;
}

// ---------------------------------------------------------------------------------------------
// precision traits
template<typename R> struct PT;
template<> struct PT<double> {
    static SKG_D double big() { return DBL_MAX; }
    static SKG_D double eps(const DevGrid& g) { return g.eps; }
};
template<> struct PT<float> {
    static SKG_D float big() { return FLT_MAX; }
    static SKG_D float eps(const DevGrid& g) { return g.epsf; }
};

template<typename R> SKG_D R gx(const DevGrid& g, int i);
template<> SKG_D double gx<double>(const DevGrid& g, int i) { return g.xv[i]; }
template<> SKG_D float  gx<float>(const DevGrid& g, int i) { return g.xvf[i]; }
template<typename R> SKG_D R gy(const DevGrid& g, int i);
template<> SKG_D double gy<double>(const DevGrid& g, int i) { return g.yv[i]; }
template<> SKG_D float  gy<float>(const DevGrid& g, int i) { return g.yvf[i]; }
template<typename R> SKG_D R gz(const DevGrid& g, int i);
template<> SKG_D double gz<double>(const DevGrid& g, int i) { return g.zv[i]; }
template<> SKG_D float  gz<float>(const DevGrid& g, int i) { return g.zvf[i]; }

// NR::locate_clip over a plane array (Fundamentals/NR.hpp:145-151)
template<typename R, R (*A)(const DevGrid&, int)>
SKG_D int locate_clip_dev(const DevGrid& g, int n /* planes */, R x) {
    if (x < A(g, 0)) return 0;
    int jl = -1, ju = n - 1;
    while (ju - jl > 1) { int jm = (ju + jl) >> 1; if (x < A(g, jm)) ju = jm; else jl = jm; }
    return jl;
}

// The (at most three) entry segments outside the grid (m = -1) that a path starts with.  Three
// named slots instead of an array: an indexed array would put the whole stepper in local memory.
template<typename R> struct Pend {
    R a, b, c;
    int n, i;
    SKG_D void clear() { n = 0; i = 0; }
    SKG_D void push(R ds) { if (n == 0) a = ds; else if (n == 1) b = ds; else c = ds; n++; }
    SKG_D bool pop(R& ds) {
        if (i >= n) return false;
        ds = (i == 0) ? a : (i == 1) ? b : c;
        i++;
        return true;
    }
};

// Resumable walks.  A stepper whose state after a cell step is fixed by a float4 (ckpt()) and the
// step count can resume() there: the walk that continues is the one that would have continued,
// step for step.  The re-walk of a path to its interaction point resumes from the last checkpoint
// of the path's own walk below the interaction optical depth instead of starting over.
// walked_from(start) is the path length from the walk's start point to the current point.
// Measured per 10^7-packet stellar phase with checkpoints every 16 steps: Voronoi traversal pass
// 1153 against 1184 ms (a cell step costs a scan of the cell's neighbour entries); the re-walk is
// 2-6 % of the cell steps of any grid (interactions lie near the start of most paths), so the
// checkpoint code in the step loop cost more than it saved for the Cartesian (74 against 69 ms)
// and lattice tree walks (k-d tree 209 against 196 ms, octree unchanged): those resume only when
// built with SKG_CKPT_CART=1 / SKG_CKPT_TREE=1.
#ifndef SKG_CKPT_CART
#define SKG_CKPT_CART 0
#endif
#ifndef SKG_CKPT_TREE
#define SKG_CKPT_TREE 0
#endif
template<class St, class = void> struct Resumable { static constexpr bool value = false; };
template<class St> struct Resumable<St, decltype((void)St::resumable, void())> {
    static constexpr bool value = St::resumable;
};

// DustGridPath::moveInside (DustGridPath.cpp:57-150).  Returns false for OUTSIDE; entry
// segments (m = -1) are appended to pd when their ds > 0.
template<typename R>
SKG_D bool move_inside(const DevGrid& g, R eps, R& rx, R& ry, R& rz, R kx, R ky, R kz, Pend<R>& pd) {
    const R xmin = (R)g.xmin, xmax = (R)g.xmax, ymin = (R)g.ymin, ymax = (R)g.ymax,
            zmin = (R)g.zmin, zmax = (R)g.zmax;
    if (rx <= xmin) {
        if (kx <= (R)0) return false;
        R ds = (xmin - rx) / kx; if (ds > (R)0) pd.push(ds);
        rx = xmin + eps; ry += ky * ds; rz += kz * ds;
    } else if (rx >= xmax) {
        if (kx >= (R)0) return false;
        R ds = (xmax - rx) / kx; if (ds > (R)0) pd.push(ds);
        rx = xmax - eps; ry += ky * ds; rz += kz * ds;
    }
    if (ry <= ymin) {
        if (ky <= (R)0) return false;
        R ds = (ymin - ry) / ky; if (ds > (R)0) pd.push(ds);
        rx += kx * ds; ry = ymin + eps; rz += kz * ds;
    } else if (ry >= ymax) {
        if (ky >= (R)0) return false;
        R ds = (ymax - ry) / ky; if (ds > (R)0) pd.push(ds);
        rx += kx * ds; ry = ymax - eps; rz += kz * ds;
    }
    if (rz <= zmin) {
        if (kz <= (R)0) return false;
        R ds = (zmin - rz) / kz; if (ds > (R)0) pd.push(ds);
        rx += kx * ds; ry += ky * ds; rz = zmin + eps;
    } else if (rz >= zmax) {
        if (kz >= (R)0) return false;
        R ds = (zmax - rz) / kz; if (ds > (R)0) pd.push(ds);
        rx += kx * ds; ry += ky * ds; rz = zmax - eps;
    }
    return true;
}

// =============================================================================================
// Cartesian: the reference's arithmetic (FP64, and the entry of the FP32 walk)
template<typename R>
struct CartStepperRef {
    R x, y, z, kx, ky, kz;
    int i, j, k;
    Pend<R> pd;
    bool done;
    int steps;
    int cell0;                  // cell holding the start position (-1 if it lies outside the grid)
    static constexpr int fallbacks = 0;
    static constexpr float rho = -1.f;   // density not embedded: the tracer reads it by cell
    SKG_D int nscanned() const { return 0; }

    // hint: a cell known to hold the start position (or -1); it is verified against the planes
    SKG_D void init(const DevGrid& g, R rx, R ry, R rz, R dx, R dy, R dz, int hint = -1) {
        x = rx; y = ry; z = rz; kx = dx; ky = dy; kz = dz;
        pd.clear(); done = false; steps = 0; cell0 = -1;
        const R xmin = (R)g.xmin, xmax = (R)g.xmax, ymin = (R)g.ymin, ymax = (R)g.ymax,
                zmin = (R)g.zmin, zmax = (R)g.zmax;
        if (hint >= 0) {
            int hi_ = hint / (g.nz * g.ny), hj = (hint / g.nz) % g.ny, hk = hint % g.nz;
            if (x >= gx<R>(g, hi_) && x <= gx<R>(g, hi_ + 1) && y >= gy<R>(g, hj) && y <= gy<R>(g, hj + 1) &&
                z >= gz<R>(g, hk) && z <= gz<R>(g, hk + 1)) {
                i = hi_; j = hj; k = hk; cell0 = hint;
                return;
            }
        }
        R ds;
        // entry into the box (CartesianDustGrid.cpp:151-222); "return path->clear()" empties the path
        if (x < xmin) {
            if (kx <= (R)0) { done = true; pd.n = 0; return; }
            ds = (xmin - x) / kx; if (ds > (R)0) pd.push(ds);
            x = xmin + (R)1e-8 * (gx<R>(g, 1) - gx<R>(g, 0)); y += ky * ds; z += kz * ds;
        } else if (x > xmax) {
            if (kx >= (R)0) { done = true; pd.n = 0; return; }
            ds = (xmax - x) / kx; if (ds > (R)0) pd.push(ds);
            x = xmax - (R)1e-8 * (gx<R>(g, g.nx) - gx<R>(g, g.nx - 1)); y += ky * ds; z += kz * ds;
        }
        if (y < ymin) {
            if (ky <= (R)0) { done = true; pd.n = 0; return; }
            ds = (ymin - y) / ky; if (ds > (R)0) pd.push(ds);
            x += kx * ds; y = ymin + (R)1e-8 * (gy<R>(g, 1) - gy<R>(g, 0)); z += kz * ds;
        } else if (y > ymax) {
            if (ky >= (R)0) { done = true; pd.n = 0; return; }
            ds = (ymax - y) / ky; if (ds > (R)0) pd.push(ds);
            x += kx * ds; y = ymax - (R)1e-8 * (gy<R>(g, g.ny) - gy<R>(g, g.ny - 1)); z += kz * ds;
        }
        if (z < zmin) {
            if (kz <= (R)0) { done = true; pd.n = 0; return; }
            ds = (zmin - z) / kz; if (ds > (R)0) pd.push(ds);
            x += kx * ds; y += ky * ds; z = zmin + (R)1e-8 * (gz<R>(g, 1) - gz<R>(g, 0));
        } else if (z > zmax) {
            if (kz >= (R)0) { done = true; pd.n = 0; return; }
            ds = (zmax - z) / kz; if (ds > (R)0) pd.push(ds);
            x += kx * ds; y += ky * ds; z = zmax - (R)1e-8 * (gz<R>(g, g.nz) - gz<R>(g, g.nz - 1));
        }
        if (x < xmin || x > xmax || y < ymin || y > ymax || z < zmin || z > zmax) { done = true; pd.n = 0; return; }
        i = locate_clip_dev<R, gx<R>>(g, g.nx + 1, x);
        j = locate_clip_dev<R, gy<R>>(g, g.ny + 1, y);
        k = locate_clip_dev<R, gz<R>>(g, g.nz + 1, z);
        if (pd.n == 0) cell0 = k + g.nz * j + g.nz * g.ny * i;
    }

    // next segment; false when the path has ended
    SKG_D bool next(const DevGrid& g, int& m, R& ds) {
        if (pd.pop(ds)) { m = -1; return true; }
        return walk(g, m, ds);
    }
    // the segments inside the grid (after the entry segments have been taken)
    SKG_D bool walk(const DevGrid& g, int& m, R& ds) {
        while (!done) {
            if (++steps > g.max_steps) { done = true; return false; }
            m = k + g.nz * j + g.nz * g.ny * i;
            R xE = (kx < (R)0) ? gx<R>(g, i) : gx<R>(g, i + 1);
            R yE = (ky < (R)0) ? gy<R>(g, j) : gy<R>(g, j + 1);
            R zE = (kz < (R)0) ? gz<R>(g, k) : gz<R>(g, k + 1);
            R dsx = (fabs(kx) > (R)1e-15) ? (xE - x) / kx : PT<R>::big();
            R dsy = (fabs(ky) > (R)1e-15) ? (yE - y) / ky : PT<R>::big();
            R dsz = (fabs(kz) > (R)1e-15) ? (zE - z) / kz : PT<R>::big();
            R d;
            if (dsx <= dsy && dsx <= dsz) {
                d = dsx;
                i += (kx < (R)0) ? -1 : 1;
                if (i >= g.nx || i < 0) done = true;
                else { x = xE; y += ky * d; z += kz * d; }
            } else if (dsy < dsx && dsy <= dsz) {
                d = dsy;
                j += (ky < (R)0) ? -1 : 1;
                if (j >= g.ny || j < 0) done = true;
                else { x += kx * d; y = yE; z += kz * d; }
            } else if (dsz < dsx && dsz < dsy) {
                d = dsz;
                k += (kz < (R)0) ? -1 : 1;
                if (k >= g.nz || k < 0) done = true;
                else { x += kx * d; y += ky * d; z = zE; }
            } else { done = true; return false; }   // NaN direction
            if (d > (R)0) { ds = d; return true; }      // DustGridPath::addSegment drops ds <= 0
        }
        return false;
    }
};

template<typename R> struct CartStepper : CartStepperRef<R> {};

// FP32 Cartesian cell step without a branch per crossed axis (1) or with the three branches (0)
#ifndef SKG_CART_SELECT
#define SKG_CART_SELECT 1
#endif

// FP32 production walk of the Cartesian grid: after the reference's entry (nudge and cell
// location), a DDA over the ray parameter t measured from the entry point.  The next wall of each
// axis sits at t = (plane - origin) / k, computed once per crossing with a reciprocal taken once per
// traversal; a segment is the difference of consecutive wall parameters (exact: Sterbenz), so no
// position is updated and nothing accumulates along the path.  Ties resolve in the reference's
// order x, y, z.
template<>
struct CartStepper<float> : CartStepperRef<float> {
    float tx, ty, tz;           // ray parameter of the next x, y and z wall
    float tc;                   // ray parameter of the current point
    float ux, uy, uz;           // 1/k (unused for an axis with |k| <= 1e-15: never crossed)

    SKG_D void init(const DevGrid& g, float rx, float ry, float rz, float dx, float dy, float dz, int hint = -1) {
        CartStepperRef<float>::init(g, rx, ry, rz, dx, dy, dz, hint);
        tc = 0.f;
        if (done) return;
        if (isnan(kx) || isnan(ky) || isnan(kz)) { done = true; return; }   // the reference walk stops
        const bool mx = fabsf(kx) > 1e-15f, my = fabsf(ky) > 1e-15f, mz = fabsf(kz) > 1e-15f;
        ux = mx ? 1.f / kx : 0.f; uy = my ? 1.f / ky : 0.f; uz = mz ? 1.f / kz : 0.f;
        tx = mx ? (gx<float>(g, kx < 0.f ? i : i + 1) - x) * ux : FLT_MAX;
        ty = my ? (gy<float>(g, ky < 0.f ? j : j + 1) - y) * uy : FLT_MAX;
        tz = mz ? (gz<float>(g, kz < 0.f ? k : k + 1) - z) * uz : FLT_MAX;
    }
    // checkpoint: the cell and the current ray parameter (the entry point and the next walls follow
    // from the start arguments)
    static constexpr bool resumable = SKG_CKPT_CART != 0;
    SKG_D float4 ckpt() const { return make_float4(__int_as_float(i), __int_as_float(j), __int_as_float(k), tc); }
    SKG_D float walked_from(float sx, float sy, float sz) const {
        return (x - sx) * kx + (y - sy) * ky + (z - sz) * kz + tc;
    }
    SKG_D void resume(const DevGrid& g, float rx, float ry, float rz, float dx, float dy, float dz, int hint, float4 c,
                      int nsteps) {
        init(g, rx, ry, rz, dx, dy, dz, hint);
        pd.clear(); steps = nsteps;
        i = __float_as_int(c.x); j = __float_as_int(c.y); k = __float_as_int(c.z); tc = c.w;
        tx = (fabsf(kx) > 1e-15f) ? (gx<float>(g, kx < 0.f ? i : i + 1) - x) * ux : FLT_MAX;
        ty = (fabsf(ky) > 1e-15f) ? (gy<float>(g, ky < 0.f ? j : j + 1) - y) * uy : FLT_MAX;
        tz = (fabsf(kz) > 1e-15f) ? (gz<float>(g, kz < 0.f ? k : k + 1) - z) * uz : FLT_MAX;
    }
    SKG_D bool next(const DevGrid& g, int& m, float& ds) {
        if (pd.pop(ds)) { m = -1; return true; }
        return walk(g, m, ds);
    }
#if SKG_CART_SELECT
    // One cell step as a single instruction stream: the crossed axis is an index and every
    // per-axis quantity a select, so lanes of a warp that cross different axes do not split into
    // three branches.  The crossed axis is the one of the three branches of the reference's tie
    // order (x if tx <= ty and tx <= tz, else y if ty <= tz, else z: for the non-NaN parameters of
    // a started walk the same choice), and every value is computed as in those branches.
    SKG_D bool walk(const DevGrid& g, int& m, float& ds) {
        while (!done) {
            if (++steps > g.max_steps) { done = true; return false; }
            m = k + g.nz * j + g.nz * g.ny * i;
            const int a = (tx <= ty && tx <= tz) ? 0 : (ty <= tz ? 1 : 2);
            const float t = a == 0 ? tx : (a == 1 ? ty : tz);
            if (t != t) { done = true; return false; }   // NaN direction
            const float ka = a == 0 ? kx : (a == 1 ? ky : kz);
            const int n = a == 0 ? g.nx : (a == 1 ? g.ny : g.nz);
            const int q = (a == 0 ? i : (a == 1 ? j : k)) + ((ka < 0.f) ? -1 : 1);
            if (a == 0) i = q;
            if (a == 1) j = q;
            if (a == 2) k = q;
            if (q >= n || q < 0) done = true;
            else {
                const float* pl = a == 0 ? g.xvf : (a == 1 ? g.yvf : g.zvf);
                const float o = a == 0 ? x : (a == 1 ? y : z);
                const float u = a == 0 ? ux : (a == 1 ? uy : uz);
                const float tn = (__ldg(pl + ((ka < 0.f) ? q : q + 1)) - o) * u;
                if (a == 0) tx = tn;
                if (a == 1) ty = tn;
                if (a == 2) tz = tn;
            }
            const float d = t - tc;
            tc = t;
            if (d > 0.f) { ds = d; return true; }   // DustGridPath::addSegment drops ds <= 0
        }
        return false;
    }
#else
    SKG_D bool walk(const DevGrid& g, int& m, float& ds) {
        while (!done) {
            if (++steps > g.max_steps) { done = true; return false; }
            m = k + g.nz * j + g.nz * g.ny * i;
            float t;
            if (tx <= ty && tx <= tz) {
                t = tx;
                i += (kx < 0.f) ? -1 : 1;
                if (i >= g.nx || i < 0) done = true;
                else tx = (gx<float>(g, kx < 0.f ? i : i + 1) - x) * ux;
            } else if (ty < tx && ty <= tz) {
                t = ty;
                j += (ky < 0.f) ? -1 : 1;
                if (j >= g.ny || j < 0) done = true;
                else ty = (gy<float>(g, ky < 0.f ? j : j + 1) - y) * uy;
            } else if (tz < tx && tz < ty) {
                t = tz;
                k += (kz < 0.f) ? -1 : 1;
                if (k >= g.nz || k < 0) done = true;
                else tz = (gz<float>(g, kz < 0.f ? k : k + 1) - z) * uz;
            } else { done = true; return false; }   // NaN direction
            const float d = t - tc;
            tc = t;
            if (d > 0.f) { ds = d; return true; }   // DustGridPath::addSegment drops ds <= 0
        }
        return false;
    }
#endif
};

// FP32 walk of a Cartesian grid whose planes are evenly spaced on every axis: the DDA of
// CartStepper<float> with the ray parameter of plane q on axis a computed as t = c0_a + q dt_a
// (c0 = (first plane - origin) / k, dt = spacing / k, fixed for a walk; one FMA) instead of loading
// the plane and selecting its table, the origin and the reciprocal by axis.  The sign of dt is the
// direction's, so the step needs no direction component either.
template<typename R> struct CartUniStepper : CartStepperRef<R> {};
template<>
struct CartUniStepper<float> : CartStepperRef<float> {
    float tx, ty, tz;           // ray parameter of the next x, y and z wall
    float tc;                   // ray parameter of the current point
    float cx, cy, cz;           // ray parameter of plane 0 per axis
    float dtx, dty, dtz;        // per plane (0 for an axis with |k| <= 1e-15: never crossed)

    SKG_D static void axis(float org, float h, float o, float k, int c, float& c0, float& dt, float& tn) {
        if (fabsf(k) > 1e-15f) {
            const float u = 1.f / k;
            c0 = (org - o) * u; dt = h * u;
            tn = fmaf((float)(k < 0.f ? c : c + 1), dt, c0);
        } else {
            c0 = 0.f; dt = 0.f; tn = FLT_MAX;
        }
    }
    SKG_D void init(const DevGrid& g, float rx, float ry, float rz, float dx, float dy, float dz, int hint = -1) {
        CartStepperRef<float>::init(g, rx, ry, rz, dx, dy, dz, hint);
        tc = 0.f;
        if (done) return;
        if (isnan(kx) || isnan(ky) || isnan(kz)) { done = true; return; }   // the reference walk stops
        axis(g.corg[0], g.cstep[0], x, kx, i, cx, dtx, tx);
        axis(g.corg[1], g.cstep[1], y, ky, j, cy, dty, ty);
        axis(g.corg[2], g.cstep[2], z, kz, k, cz, dtz, tz);
    }
    static constexpr bool resumable = false;
    SKG_D bool next(const DevGrid& g, int& m, float& ds) {
        if (pd.pop(ds)) { m = -1; return true; }
        return walk(g, m, ds);
    }
    // one cell step: the crossed axis (the reference's tie order) and every per-axis value a select
    SKG_D bool walk(const DevGrid& g, int& m, float& ds) {
        while (!done) {
            if (++steps > g.max_steps) { done = true; return false; }
            m = k + g.nz * j + g.nz * g.ny * i;
            const int a = (tx <= ty && tx <= tz) ? 0 : (ty <= tz ? 1 : 2);
            const float t = a == 0 ? tx : (a == 1 ? ty : tz);
            if (t != t) { done = true; return false; }   // NaN direction
            const float dt = a == 0 ? dtx : (a == 1 ? dty : dtz);
            const bool neg = dt < 0.f;
            const int n = a == 0 ? g.nx : (a == 1 ? g.ny : g.nz);
            const int q = (a == 0 ? i : (a == 1 ? j : k)) + (neg ? -1 : 1);
            if (a == 0) i = q;
            if (a == 1) j = q;
            if (a == 2) k = q;
            if (q >= n || q < 0) done = true;
            else {
                const float c0 = a == 0 ? cx : (a == 1 ? cy : cz);
                const float tn = fmaf((float)(neg ? q : q + 1), dt, c0);
                if (a == 0) tx = tn;
                if (a == 1) ty = tn;
                if (a == 2) tz = tn;
            }
            const float d = t - tc;
            tc = t;
            if (d > 0.f) { ds = d; return true; }   // DustGridPath::addSegment drops ds <= 0
        }
        return false;
    }
};

// =============================================================================================
// Tree (octree and k-d tree)
template<typename R> SKG_D void node_bounds(const DevGrid& g, int l, V3<R>& lo, V3<R>& hi);
template<> SKG_D void node_bounds<double>(const DevGrid& g, int l, V3<double>& lo, V3<double>& hi) {
    const double* b = g.node_box + 6 * (size_t)l;
    lo = mk3(b[0], b[1], b[2]); hi = mk3(b[3], b[4], b[5]);
}
template<> SKG_D void node_bounds<float>(const DevGrid& g, int l, V3<float>& lo, V3<float>& hi) {
    float4 a = __ldg(g.nodef + 2 * (size_t)l), b = __ldg(g.nodef + 2 * (size_t)l + 1);
    lo = mk3(a.x, a.y, a.z); hi = mk3(b.x, b.y, b.z);
}
template<typename R> SKG_D V3<R> node_hi(const DevGrid& g, int l);
template<> SKG_D V3<double> node_hi<double>(const DevGrid& g, int l) {
    const double* b = g.node_box + 6 * (size_t)l; return mk3(b[3], b[4], b[5]);
}
template<> SKG_D V3<float> node_hi<float>(const DevGrid& g, int l) {
    float4 b = __ldg(g.nodef + 2 * (size_t)l + 1); return mk3(b.x, b.y, b.z);
}
template<typename R> SKG_D bool box_contains(V3<R> lo, V3<R> hi, R x, R y, R z) {   // Box.hpp:80-81
    return x >= lo.x && x <= hi.x && y >= lo.y && y <= hi.y && z >= lo.z && z <= hi.z;
}

// TreeNode::child(r): OctTreeNode.cpp:184-189 / BinTreeNode.cpp:326-335
template<typename R>
SKG_D int tree_child(const DevGrid& g, int l, R x, R y, R z) {
    int c0 = g.node_child[l];
    V3<R> s = node_hi<R>(g, c0);
    int d = g.node_dir[l];
    if (d < 0) return c0 + (x < s.x ? 0 : 1) + (y < s.y ? 0 : 2) + (z < s.z ? 0 : 4);
    if (d == 0) return x < s.x ? c0 : c0 + 1;
    if (d == 1) return y < s.y ? c0 : c0 + 1;
    return z < s.z ? c0 : c0 + 1;
}
// TreeNode::whichnode from the root (TreeNode.cpp:70-80)
template<typename R>
SKG_D int tree_whichnode(const DevGrid& g, R x, R y, R z) {
    V3<R> lo, hi; node_bounds<R>(g, 0, lo, hi);
    if (!box_contains(lo, hi, x, y, z)) return -1;
    int l = 0;
    int guard = 0;
    while (g.node_child[l] >= 0 && guard++ < 64) l = tree_child<R>(g, l, x, y, z);
    return l;
}

template<typename R>
struct TreeNodeWalk {
    R x, y, z, kx, ky, kz;
    int node;
    Pend<R> pd;
    bool done;
    int steps;
    int fallbacks;
    int scanned;
    SKG_D int nscanned() const { return scanned; }
    int cell0;
    static constexpr float rho = -1.f;

    SKG_D void init(const DevGrid& g, R rx, R ry, R rz, R dx, R dy, R dz, int hint = -1) {
        kx = dx; ky = dy; kz = dz; pd.clear(); done = false; steps = 0; fallbacks = 0; scanned = 0;
        cell0 = -1;
        if (hint >= 0) {
            int l = g.cell_node[hint];
            V3<R> lo, hi; node_bounds<R>(g, l, lo, hi);
            if (box_contains(lo, hi, rx, ry, rz)) { node = l; x = rx; y = ry; z = rz; cell0 = hint; return; }
        }
        R eps = PT<R>::eps(g);
        bool ok = move_inside<R>(g, eps, rx, ry, rz, kx, ky, kz, pd);
        node = ok ? tree_whichnode<R>(g, rx, ry, rz) : -1;
        if (node < 0) { pd.n = 0; done = true; return; }   // path->clear()
        if (pd.n == 0) cell0 = g.node_cell[node];
        x = rx; y = ry; z = rz;
    }

    SKG_D bool next(const DevGrid& g, int& m, R& ds) {
        if (pd.pop(ds)) { m = -1; return true; }
        return walk(g, m, ds);
    }
    // the segments inside the grid (after the entry segments have been taken)
    SKG_D bool walk(const DevGrid& g, int& m, R& ds) {
        while (!done) {
            if (++steps > g.max_steps) { done = true; return false; }
            if (g.search == 2) { if (bookkeeping(g, m, ds)) return true; else continue; }
            V3<R> lo, hi; node_bounds<R>(g, node, lo, hi);
            R xnext = (kx < (R)0) ? lo.x : hi.x;
            R ynext = (ky < (R)0) ? lo.y : hi.y;
            R znext = (kz < (R)0) ? lo.z : hi.z;
            R dsx = (fabs(kx) > (R)1e-15) ? (xnext - x) / kx : PT<R>::big();
            R dsy = (fabs(ky) > (R)1e-15) ? (ynext - y) / ky : PT<R>::big();
            R dsz = (fabs(kz) > (R)1e-15) ? (znext - z) / kz : PT<R>::big();
            R d; int wall;
            if (dsx <= dsy && dsx <= dsz) { d = dsx; wall = (kx < (R)0) ? 0 : 1; }
            else if (dsy <= dsx && dsy <= dsz) { d = dsy; wall = (ky < (R)0) ? 2 : 3; }
            else { d = dsz; wall = (kz < (R)0) ? 4 : 5; }
            m = g.node_cell[node];
            R eps = PT<R>::eps(g);
            x += (d + eps) * kx; y += (d + eps) * ky; z += (d + eps) * kz;
            int oldnode = node;
            if (g.search == 1) {
                int found = -1;
                int q1 = g.nbroff[6 * node + wall + 1];
                for (int q = g.nbroff[6 * node + wall]; q < q1; q++) {
                    int c = __ldg(g.nbr + q);
                    scanned++;
                    V3<R> l2, h2; node_bounds<R>(g, c, l2, h2);
                    if (box_contains(l2, h2, x, y, z)) { found = c; break; }
                }
                if (found < 0) { found = tree_whichnode<R>(g, x, y, z); fallbacks++; }
                node = found;
            } else {
                node = tree_whichnode<R>(g, x, y, z);
            }
            if (node == oldnode) {      // TreeDustGrid.cpp:418-435
                x = nextafter(x, (kx < (R)0) ? -PT<R>::big() : PT<R>::big());
                y = nextafter(y, (ky < (R)0) ? -PT<R>::big() : PT<R>::big());
                z = nextafter(z, (kz < (R)0) ? -PT<R>::big() : PT<R>::big());
                node = tree_whichnode<R>(g, x, y, z);
                if (node == oldnode) node = -1;
            }
            if (node < 0) done = true;
            // FP32: the nudge past the wall is credited to this segment so that the total path
            // length stays exact (FP64 keeps the reference's accounting)
            if (sizeof(R) == 4 && node >= 0) d += eps;
            if (d > (R)0) { ds = d; return true; }
        }
        return false;
    }

    // Bookkeeping search (TreeDustGrid.cpp:500-640), octree only: neighbour found by index
    // arithmetic over siblings and fathers.  Returns true when a segment was produced.
    SKG_D bool bookkeeping(const DevGrid& g, int& m, R& ds) {
        int l = node;
        V3<R> lo, hi; node_bounds<R>(g, l, lo, hi);
        R xnext = (kx < (R)0) ? lo.x : hi.x;
        R ynext = (ky < (R)0) ? lo.y : hi.y;
        R znext = (kz < (R)0) ? lo.z : hi.z;
        R dsx = (fabs(kx) > (R)1e-15) ? (xnext - x) / kx : PT<R>::big();
        R dsy = (fabs(ky) > (R)1e-15) ? (ynext - y) / ky : PT<R>::big();
        R dsz = (fabs(kz) > (R)1e-15) ? (znext - z) / kz : PT<R>::big();
        R d;
        m = g.node_cell[l];
        if (dsx <= dsy && dsx <= dsz) {
            d = dsx; x = xnext; y += ky * d; z += kz * d;
            while (true) {
                int oct = ((l - 1) % 8) + 1;
                bool place = (kx < (R)0) ? (oct % 2 == 1) : (oct % 2 == 0);
                if (!place) break;
                l = g.node_father[l];
                if (l == 0) { done = true; break; }
            }
            if (!done) {
                l += (kx < (R)0) ? -1 : 1;
                while (g.node_cell[l] == -1) {
                    int c0 = g.node_child[l]; V3<R> s = node_hi<R>(g, c0);
                    if (kx < (R)0) l = (y <= s.y) ? ((z <= s.z) ? c0 + 1 : c0 + 5) : ((z <= s.z) ? c0 + 3 : c0 + 7);
                    else           l = (y <= s.y) ? ((z <= s.z) ? c0 + 0 : c0 + 4) : ((z <= s.z) ? c0 + 2 : c0 + 6);
                }
            }
        } else if (dsy < dsx && dsy <= dsz) {
            d = dsy; x += kx * d; y = ynext; z += kz * d;
            while (true) {
                bool place = (ky < (R)0) ? ((l - 1) % 4 < 2) : ((l - 1) % 4 > 1);
                if (!place) break;
                l = g.node_father[l];
                if (l == 0) { done = true; break; }
            }
            if (!done) {
                l += (ky < (R)0) ? -2 : 2;
                while (g.node_cell[l] == -1) {
                    int c0 = g.node_child[l]; V3<R> s = node_hi<R>(g, c0);
                    if (ky < (R)0) l = (x <= s.x) ? ((z <= s.z) ? c0 + 2 : c0 + 6) : ((z <= s.z) ? c0 + 3 : c0 + 7);
                    else           l = (x <= s.x) ? ((z <= s.z) ? c0 + 0 : c0 + 4) : ((z <= s.z) ? c0 + 1 : c0 + 5);
                }
            }
        } else if (dsz < dsx && dsz < dsy) {
            d = dsz; x += kx * d; y += ky * d; z = znext;
            while (true) {
                int oct = ((l - 1) % 8) + 1;
                bool place = (kz < (R)0) ? (oct < 5) : (oct > 4);
                if (!place) break;
                l = g.node_father[l];
                if (l == 0) { done = true; break; }
            }
            if (!done) {
                l += (kz < (R)0) ? -4 : 4;
                while (g.node_cell[l] == -1) {
                    int c0 = g.node_child[l]; V3<R> s = node_hi<R>(g, c0);
                    if (kz < (R)0) l = (x <= s.x) ? ((y <= s.y) ? c0 + 4 : c0 + 6) : ((y <= s.y) ? c0 + 5 : c0 + 7);
                    else           l = (x <= s.x) ? ((y <= s.y) ? c0 + 0 : c0 + 2) : ((y <= s.y) ? c0 + 1 : c0 + 3);
                }
            }
        } else { done = true; return false; }
        node = l;
        if (d > (R)0) { ds = d; return true; }
        return false;
    }
};

// FP32 production walk of the tree (the cells of TreeDustGrid.cpp:443-497, Neighbor or TopDown
// search): the current leaf's 64-byte record stays in registers; a step follows the rope of the
// exit wall and descends from it through the internal records to the leaf holding the new point,
// whose record becomes the current one.  FP64 walks and the Bookkeeping search run through the
// node-based walk above (the launchers pick TreeNodeWalk<float> for Bookkeeping).
template<typename R> struct TreeStepper : TreeNodeWalk<R> {};

template<>
struct TreeStepper<float> {
    float x, y, z, kx, ky, kz;
    float4 r0, r1;              // the current leaf's box, density and cell (its ropes stay in L1)
    int leaf;
    Pend<float> pd;
    bool done;
    int steps, fallbacks;
    SKG_D int nscanned() const { return steps; }   // one rope followed per step
    int cell0;
    float rho;                  // density embedded in the record of the last segment's cell

    SKG_D void load(const DevGrid& g, int li) {
        const float4* p = g.lrec + 4 * (size_t)li;
        r0 = __ldg(p); r1 = __ldg(p + 1);
    }
    SKG_D bool inside(float px, float py, float pz) const {
        return px >= r0.x && px <= r1.x && py >= r0.y && py <= r1.y && pz >= r0.z && pz <= r1.z;
    }
    // descends from a node reference to the leaf holding the point (the reference's child(r)
    // rule: a point on a split plane belongs to the upper child)
    SKG_D static int descend(const DevGrid& g, int ref, float px, float py, float pz) {
        int guard = 0;
        while (ref < -1 && guard++ < 64) {
            // the split point and both child-reference vectors in one round trip (one 48-byte record)
            const float4* p = g.irec + 3 * (size_t)(-ref - 2);
            const float4 a = __ldg(p), b0 = __ldg(p + 1), b1 = __ldg(p + 2);
            int d = __float_as_int(a.w), c;
            if (d < 0) c = (px < a.x ? 0 : 1) + (py < a.y ? 0 : 2) + (pz < a.z ? 0 : 4);
            else c = ((d == 0 ? px < a.x : d == 1 ? py < a.y : pz < a.z) ? 0 : 1);
            const float4 b = (c >> 2) ? b1 : b0;
            int k = c & 3;
            ref = __float_as_int(k == 0 ? b.x : k == 1 ? b.y : k == 2 ? b.z : b.w);
        }
        return ref;
    }
    SKG_D static int locate(const DevGrid& g, float px, float py, float pz) {
        if (!(px >= (float)g.xmin && px <= (float)g.xmax && py >= (float)g.ymin && py <= (float)g.ymax &&
              pz >= (float)g.zmin && pz <= (float)g.zmax)) return -1;
        return descend(g, g.root_ref, px, py, pz);
    }

    SKG_D void init(const DevGrid& g, float rx, float ry, float rz, float dx, float dy, float dz, int hint = -1) {
        kx = dx; ky = dy; kz = dz; pd.clear(); done = false; steps = 0; fallbacks = 0;
        cell0 = -1; rho = -1.f;
        if (hint >= 0) {
            leaf = __ldg(g.cell_leaf + hint);
            load(g, leaf);
            if (inside(rx, ry, rz)) { cell0 = hint; x = rx; y = ry; z = rz; return; }
        }
        bool ok = move_inside<float>(g, g.epsf, rx, ry, rz, kx, ky, kz, pd);
        leaf = ok ? locate(g, rx, ry, rz) : -1;
        if (leaf < 0) { pd.n = 0; done = true; return; }
        load(g, leaf);
        if (pd.n == 0) cell0 = __float_as_int(r1.w);
        x = rx; y = ry; z = rz;
    }

    SKG_D bool next(const DevGrid& g, int& m, float& ds) {
        if (pd.pop(ds)) { m = -1; rho = 0.f; return true; }
        return walk(g, m, ds);
    }
    // the segments inside the grid (after the entry segments have been taken)
    SKG_D bool walk(const DevGrid& g, int& m, float& ds) {
        const float eps = g.epsf;
        while (!done) {
            if (++steps > g.max_steps) { done = true; return false; }
            float xnext = (kx < 0.f) ? r0.x : r1.x;
            float ynext = (ky < 0.f) ? r0.y : r1.y;
            float znext = (kz < 0.f) ? r0.z : r1.z;
            float dsx = (fabsf(kx) > 1e-15f) ? (xnext - x) / kx : FLT_MAX;
            float dsy = (fabsf(ky) > 1e-15f) ? (ynext - y) / ky : FLT_MAX;
            float dsz = (fabsf(kz) > 1e-15f) ? (znext - z) / kz : FLT_MAX;
            float d; int face;          // exit wall: 0..5 = x-, x+, y-, y+, z-, z+
            if (dsx <= dsy && dsx <= dsz) { d = dsx; face = (kx < 0.f) ? 0 : 1; }
            else if (dsy <= dsx && dsy <= dsz) { d = dsy; face = (ky < 0.f) ? 2 : 3; }
            else { d = dsz; face = (kz < 0.f) ? 4 : 5; }
            // the rope of that wall: words 8..13 of the leaf's record (the line is in L1)
            const int rope = __ldg(reinterpret_cast<const int*>(g.lrec + 4 * (size_t)leaf + 2) + face);
            m = __float_as_int(r1.w);
            rho = r0.w;
            x += (d + eps) * kx; y += (d + eps) * ky; z += (d + eps) * kz;
            // follow the rope of the exit wall; if the point is not in the leaf it leads to (it
            // crossed near an edge or corner), locate it from the root
            int next = (rope == -1) ? -1 : descend(g, rope, x, y, z);
            if (next >= 0) {
                load(g, next);
                if (!inside(x, y, z)) {
                    next = locate(g, x, y, z); fallbacks++;
                    if (next >= 0) load(g, next);
                }
            } else if (rope != -1) {
                next = locate(g, x, y, z); fallbacks++;
                if (next >= 0) load(g, next);
            }
            if (next == leaf) {                    // stuck (TreeDustGrid.cpp:476-493)
                x = nextafterf(x, (kx < 0.f) ? -FLT_MAX : FLT_MAX);
                y = nextafterf(y, (ky < 0.f) ? -FLT_MAX : FLT_MAX);
                z = nextafterf(z, (kz < 0.f) ? -FLT_MAX : FLT_MAX);
                next = locate(g, x, y, z);
                if (next == leaf) next = -1;
                else if (next >= 0) load(g, next);
            }
            if (next < 0) done = true;
            else { leaf = next; d += eps; }      // the nudge is credited to the segment left behind
            if (d > 0.f) { ds = d; return true; }
        }
        return false;
    }
};

// FP32 walk on the lattice form of the rope tree: the same steps as TreeStepper<float>, with the
// current leaf's 32-byte record (density, centre codes, packed ropes) in registers and its walls
// computed from the codes.  A leaf reference is the cell number.
// reciprocal directions for the exit distances of the lattice walk: the traversal kernels are
// issue-bound, and three multiplies replace three IEEE divisions per cell step (octree disk,
// traversal pass 164 against 170 ms per 10^7 packets)
#ifndef SKG_LAT_RCP
#define SKG_LAT_RCP 1
#endif
// whether the nudged point crossed the exit face's interior, from the positions (0: six compares
// and three selects) or from the exit distances (1: three compares); near an edge the two can
// round differently, and a point that lands a rounding error outside its leaf steps on with a
// dropped non-positive segment.  Traversal pass of a 10^7-packet phase: octree disk 1283 against
// 1360 ms, k-d tree disk 1669 against 1717 ms; 10 of 1.29·10^11 cell steps differ on the octree
#ifndef SKG_LAT_DS_FACE
#define SKG_LAT_DS_FACE 1
#endif
// the exit wall's rope taken per axis (1) or by its bit position (0); the same bits (traversal pass
// of a 10^7-packet phase: octree disk 1364 against 1441 ms, k-d tree disk 1725 against 1791 ms)
#ifndef SKG_LAT_AXIS_ROPE
#define SKG_LAT_AXIS_ROPE 1
#endif
template<typename R> struct TreeLatticeStepper : TreeNodeWalk<R> {};

template<>
struct TreeLatticeStepper<float> {
    float x, y, z, kx, ky, kz;
#if SKG_LAT_RCP
    float ux, uy, uz;           // 1/k per axis (0 where |k| <= 1e-15: that axis is never crossed)
#endif
    uint4 a, b;                 // the current leaf's record
    int leaf;                   // its cell number
    Pend<float> pd;
    bool done;
    int steps, fallbacks;
    SKG_D int nscanned() const { return steps; }   // one rope followed per step
    int cell0;
    float rho;

    SKG_D void load(const DevGrid& g, int li) {
        const uint4* p = g.prec + 2 * (size_t)li;
        a = __ldg(p); b = __ldg(p + 1);
    }
    SKG_D static uint32_t code_x(const uint4& a) { return a.y & 0x1FFFFFu; }
    SKG_D static uint32_t code_y(const uint4& a) { return __funnelshift_r(a.y, a.z, 21) & 0x1FFFFFu; }
    SKG_D static uint32_t code_z(const uint4& a) { return (a.z >> 10) & 0x1FFFFFu; }
    // the low (up = false) or high wall of the interval with centre code c
    SKG_D static float wall(uint32_t c, bool up, float org, float unit) {
        const uint32_t t = c & (0u - c);          // half the width: the code's lowest set bit
        return fmaf((float)(up ? c + t : c - t), unit, org);
    }
    SKG_D static bool within(uint32_t c, float p, float org, float unit) {
        const uint32_t t = c & (0u - c);
        return p >= fmaf((float)(c - t), unit, org) && p <= fmaf((float)(c + t), unit, org);
    }
    SKG_D bool inside(const DevGrid& g, float px, float py, float pz) const {
        return within(code_x(a), px, g.lorg[0], g.lunit[0]) && within(code_y(a), py, g.lorg[1], g.lunit[1]) &&
               within(code_z(a), pz, g.lorg[2], g.lunit[2]);
    }
    // decoded rope: -1 the outside, a cell number, or an internal record as -(index) - 2
    SKG_D static int rope_ref(uint32_t v) {
        v &= 0x3FFFFFFu;
        return v == 0x3FFFFFFu ? -1 : (v >= (1u << 25)) ? -(int)(v - (1u << 25)) - 2 : (int)v;
    }
    // the rope of the exit wall on axis ax (its side given by the walk's direction): the word pair
    // and the shift of each axis's exit wall are fixed for a walk, so a step takes three funnel
    // shifts and two selects instead of selecting words by a computed bit position
    SKG_D int exit_rope(int ax) const {
        const uint32_t rx = __funnelshift_r(a.w, b.x, kx < 0.f ? 0 : 26);
        const uint32_t ry = ky < 0.f ? __funnelshift_r(b.x, b.y, 20) : __funnelshift_r(b.y, b.z, 14);
        const uint32_t rz = kz < 0.f ? __funnelshift_r(b.z, b.w, 8) : (b.w >> 2);
        return rope_ref(ax == 0 ? rx : ax == 1 ? ry : rz);
    }
    // the reference of wall f: 26 bits at bit 26 f of the 160-bit string (a.w, b.x, b.y, b.z, b.w)
    SKG_D int rope(int f) const {
        const int bit = 26 * f, wd = bit >> 5, sh = bit & 31;
        const uint32_t lo = wd == 0 ? a.w : wd == 1 ? b.x : wd == 2 ? b.y : wd == 3 ? b.z : b.w;
        const uint32_t hi = wd == 0 ? b.x : wd == 1 ? b.y : wd == 2 ? b.z : b.w;
        const uint32_t v = __funnelshift_r(lo, hi, sh) & 0x3FFFFFFu;
        return v == 0x3FFFFFFu ? -1 : (v >= (1u << 25)) ? -(int)(v - (1u << 25)) - 2 : (int)v;
    }

    SKG_D void set_dir(float dx, float dy, float dz) {
        kx = dx; ky = dy; kz = dz; pd.clear(); done = false; steps = 0; fallbacks = 0;
        cell0 = -1; rho = -1.f;
#if SKG_LAT_RCP
        ux = (fabsf(kx) > 1e-15f) ? 1.f / kx : 0.f;
        uy = (fabsf(ky) > 1e-15f) ? 1.f / ky : 0.f;
        uz = (fabsf(kz) > 1e-15f) ? 1.f / kz : 0.f;
#endif
    }
    // checkpoint: the position and the current leaf
    static constexpr bool resumable = SKG_CKPT_TREE != 0;
    SKG_D float4 ckpt() const { return make_float4(x, y, z, __int_as_float(leaf)); }
    SKG_D float walked_from(float sx, float sy, float sz) const { return (x - sx) * kx + (y - sy) * ky + (z - sz) * kz; }
    SKG_D void resume(const DevGrid& g, float, float, float, float dx, float dy, float dz, int, float4 c, int nsteps) {
        set_dir(dx, dy, dz);
        steps = nsteps;
        x = c.x; y = c.y; z = c.z; leaf = __float_as_int(c.w);
        load(g, leaf);
    }

    SKG_D void init(const DevGrid& g, float rx, float ry, float rz, float dx, float dy, float dz, int hint = -1) {
        set_dir(dx, dy, dz);
        if (hint >= 0) {
            leaf = hint;
            load(g, leaf);
            if (inside(g, rx, ry, rz)) { cell0 = hint; x = rx; y = ry; z = rz; return; }
        }
        bool ok = move_inside<float>(g, g.epsf, rx, ry, rz, kx, ky, kz, pd);
        leaf = ok ? TreeStepper<float>::locate(g, rx, ry, rz) : -1;
        if (leaf < 0) { pd.n = 0; done = true; return; }
        load(g, leaf);
        if (pd.n == 0) cell0 = leaf;
        x = rx; y = ry; z = rz;
    }

    SKG_D bool next(const DevGrid& g, int& m, float& ds) {
        if (pd.pop(ds)) { m = -1; rho = 0.f; return true; }
        return walk(g, m, ds);
    }
    SKG_D bool walk(const DevGrid& g, int& m, float& ds) {
        const float eps = g.epsf;
        while (!done) {
            if (++steps > g.max_steps) { done = true; return false; }
            const float xnext = wall(code_x(a), kx >= 0.f, g.lorg[0], g.lunit[0]);
            const float ynext = wall(code_y(a), ky >= 0.f, g.lorg[1], g.lunit[1]);
            const float znext = wall(code_z(a), kz >= 0.f, g.lorg[2], g.lunit[2]);
#if SKG_LAT_RCP
            // exit distances with the traversal's reciprocal directions: within an ulp of the
            // quotients, far inside the 4-ulp nudge past each wall
            float dsx = (ux != 0.f) ? (xnext - x) * ux : FLT_MAX;
            float dsy = (uy != 0.f) ? (ynext - y) * uy : FLT_MAX;
            float dsz = (uz != 0.f) ? (znext - z) * uz : FLT_MAX;
#else
            float dsx = (fabsf(kx) > 1e-15f) ? (xnext - x) / kx : FLT_MAX;
            float dsy = (fabsf(ky) > 1e-15f) ? (ynext - y) / ky : FLT_MAX;
            float dsz = (fabsf(kz) > 1e-15f) ? (znext - z) / kz : FLT_MAX;
#endif
            float d; int face;          // exit wall: 0..5 = x-, x+, y-, y+, z-, z+
            if (dsx <= dsy && dsx <= dsz) { d = dsx; face = (kx < 0.f) ? 0 : 1; }
            else if (dsy <= dsx && dsy <= dsz) { d = dsy; face = (ky < 0.f) ? 2 : 3; }
            else { d = dsz; face = (kz < 0.f) ? 4 : 5; }
#if SKG_LAT_AXIS_ROPE
            const int rp = exit_rope(face >> 1);
#else
            const int rp = rope(face);
#endif
            m = leaf;
            rho = __uint_as_float(a.x);
            x += (d + eps) * kx; y += (d + eps) * ky; z += (d + eps) * kz;
            // The rope's node covers the whole exit face: when the point lies beyond (or on) the
            // exit wall and, along the other axes, still within the walls ahead of it, the leaf it
            // descends to holds it and the containment test can be skipped (the point crossed
            // near an edge or a corner otherwise).
            const int ax = face >> 1;
#if SKG_LAT_DS_FACE
            // the same question asked of the exit distances: the point moved d + eps along the ray,
            // so it stays within the other axes' walls ahead when those are at least that far
            const float lim = d + eps;
            const bool on_face = (ax == 0 || dsx >= lim) && (ax == 1 || dsy >= lim) && (ax == 2 || dsz >= lim);
#else
            const bool bx = (kx < 0.f) ? (x <= xnext) : (x >= xnext), wx = (kx < 0.f) ? (x >= xnext) : (x <= xnext);
            const bool by = (ky < 0.f) ? (y <= ynext) : (y >= ynext), wy = (ky < 0.f) ? (y >= ynext) : (y <= ynext);
            const bool bz = (kz < 0.f) ? (z <= znext) : (z >= znext), wz = (kz < 0.f) ? (z >= znext) : (z <= znext);
            const bool on_face = (ax == 0 ? bx : wx) && (ax == 1 ? by : wy) && (ax == 2 ? bz : wz);
#endif
            int next = (rp == -1) ? -1 : TreeStepper<float>::descend(g, rp, x, y, z);
            if (next >= 0) {
                load(g, next);
                if (!on_face && !inside(g, x, y, z)) {
                    next = TreeStepper<float>::locate(g, x, y, z); fallbacks++;
                    if (next >= 0) load(g, next);
                }
            } else if (rp != -1) {
                next = TreeStepper<float>::locate(g, x, y, z); fallbacks++;
                if (next >= 0) load(g, next);
            }
            if (next == leaf) {                    // stuck (TreeDustGrid.cpp:476-493)
                x = nextafterf(x, (kx < 0.f) ? -FLT_MAX : FLT_MAX);
                y = nextafterf(y, (ky < 0.f) ? -FLT_MAX : FLT_MAX);
                z = nextafterf(z, (kz < 0.f) ? -FLT_MAX : FLT_MAX);
                next = TreeStepper<float>::locate(g, x, y, z);
                if (next == leaf) next = -1;
                else if (next >= 0) load(g, next);
            }
            if (next < 0) done = true;
            else { leaf = next; d += eps; }
            if (d > 0.f) { ds = d; return true; }
        }
        return false;
    }
};

// =============================================================================================
// Voronoi
#ifndef SKG_VOR_NODIV
#define SKG_VOR_NODIV 1
#endif
template<typename R> SKG_D V3<R> site_pos(const DevGrid& g, int m);
template<> SKG_D V3<double> site_pos<double>(const DevGrid& g, int m) {
    const double* p = g.site + 3 * (size_t)m; return mk3(p[0], p[1], p[2]);
}
template<> SKG_D V3<float> site_pos<float>(const DevGrid& g, int m) {
    float4 p = __ldg(g.sitef + m); return mk3(p.x, p.y, p.z);
}

// VoronoiMesh::cellIndex (VoronoiMesh.cpp:541-570): nearest site among the cells overlapping the
// block of the point (the reference's per-block kd-tree is an exact nearest search).
template<typename R>
SKG_D int voronoi_cell_index(const DevGrid& g, R x, R y, R z) {
    if (!(x >= (R)g.xmin && x <= (R)g.xmax && y >= (R)g.ymin && y <= (R)g.ymax &&
          z >= (R)g.zmin && z <= (R)g.zmax)) return -1;
    int nb = g.nb;
    // Box::cellindices (Box.hpp:120-125) evaluated in double
    int i = max(0, min(nb - 1, (int)(nb * ((double)x - g.xmin) / (g.xmax - g.xmin))));
    int j = max(0, min(nb - 1, (int)(nb * ((double)y - g.ymin) / (g.ymax - g.ymin))));
    int k = max(0, min(nb - 1, (int)(nb * ((double)z - g.zmin) / (g.zmax - g.zmin))));
    int b = (i * nb + j) * nb + k;
    // squared distances in FP64 for both precisions (they overflow FP32 for galaxy-sized domains)
    int m = -1; double mdist = DBL_MAX;
    int q1 = g.boff[b + 1];
    for (int q = g.boff[b]; q < q1; q++) {
        int id = __ldg(g.bids + q);
        V3<double> p = site_pos<double>(g, id);
        double dx = (double)x - p.x, dy = (double)y - p.y, dz = (double)z - p.z;
        double d = dx * dx + dy * dy + dz * dz;
        if (d < mdist) { m = id; mdist = d; }
    }
    return m;
}

template<typename R>
struct VoronoiStepper {
    R x, y, z, kx, ky, kz;
    int mr;
    int qb, qe;                 // neighbour entries of the current cell (FP32 walk; qe < 0: not read yet)
    Pend<R> pd;
    bool done;
    int steps;
    int fallbacks;
    int scanned;
    SKG_D int nscanned() const { return scanned; }
    int cell0;
    static constexpr float rho = -1.f;

    // hint: the cell holding the start position (the interaction point lies in the cell of its
    // segment); accepted for a position strictly inside the domain
    SKG_D void init(const DevGrid& g, R rx, R ry, R rz, R dx, R dy, R dz, int hint = -1) {
        kx = dx; ky = dy; kz = dz; pd.clear(); done = false; steps = 0; fallbacks = 0; scanned = 0;
        cell0 = -1; qb = 0; qe = -1;
        if (hint >= 0 && rx > (R)g.xmin && rx < (R)g.xmax && ry > (R)g.ymin && ry < (R)g.ymax &&
            rz > (R)g.zmin && rz < (R)g.zmax) {
            mr = hint; cell0 = hint; x = rx; y = ry; z = rz;
            return;
        }
        R eps = PT<R>::eps(g);
        bool ok = move_inside<R>(g, eps, rx, ry, rz, kx, ky, kz, pd);
        if (!ok) { rx = ry = rz = (R)INFINITY; }
        mr = voronoi_cell_index<R>(g, rx, ry, rz);
        if (mr < 0) { pd.n = 0; done = true; return; }
        if (pd.n == 0) cell0 = mr;
        x = rx; y = ry; z = rz;
    }

    // checkpoint of the FP32 walk: the position and the current cell (its neighbour entries are
    // read again from the CSR offsets, the values the walk carried)
    static constexpr bool resumable = std::is_same<R, float>::value;
    SKG_D float4 ckpt() const { return make_float4((float)x, (float)y, (float)z, __int_as_float(mr)); }
    SKG_D float walked_from(float sx, float sy, float sz) const {
        return ((float)x - sx) * (float)kx + ((float)y - sy) * (float)ky + ((float)z - sz) * (float)kz;
    }
    SKG_D void resume(const DevGrid& g, R, R, R, R dx, R dy, R dz, int, float4 c, int nsteps) {
        kx = dx; ky = dy; kz = dz; pd.clear(); done = false; steps = nsteps; fallbacks = 0; scanned = 0;
        cell0 = -1; qb = 0; qe = -1;
        x = (R)c.x; y = (R)c.y; z = (R)c.z; mr = __float_as_int(c.w);
    }

    SKG_D bool next(const DevGrid& g, int& m, R& ds) {
        if (pd.pop(ds)) { m = -1; return true; }
        return walk(g, m, ds);
    }
    // the segments inside the grid (after the entry segments have been taken)
    SKG_D bool walk(const DevGrid& g, int& m, R& ds);
};

// FP64: the reference arithmetic on the generator sites (VoronoiMesh.cpp:803-858)
template<>
SKG_D bool VoronoiStepper<double>::walk(const DevGrid& g, int& m, double& ds) {
    while (!done) {
        if (++steps > g.max_steps) { done = true; return false; }
        V3<double> pr = site_pos<double>(g, mr);
        double sq = DBL_MAX;
        int mq = -99;
        int q1 = g.vnoff[mr + 1];
        for (int q = g.vnoff[mr]; q < q1; q++) {
            int mi = g.vnbr[q];
            double si = 0;
            scanned++;
            if (mi >= 0) {
                V3<double> pi = site_pos<double>(g, mi);
                double nx = pi.x - pr.x, ny = pi.y - pr.y, nz = pi.z - pr.z;
                double ndotk = nx * kx + ny * ky + nz * kz;
                if (ndotk > 0) {
                    double px = 0.5 * (pi.x + pr.x), py = 0.5 * (pi.y + pr.y), pz = 0.5 * (pi.z + pr.z);
                    si = (nx * (px - x) + ny * (py - y) + nz * (pz - z)) / ndotk;
                }
            } else {
                switch (mi) {
                    case -1: si = (g.xmin - x) / kx; break;
                    case -2: si = (g.xmax - x) / kx; break;
                    case -3: si = (g.ymin - y) / ky; break;
                    case -4: si = (g.ymax - y) / ky; break;
                    case -5: si = (g.zmin - z) / kz; break;
                    default: si = (g.zmax - z) / kz; break;
                }
            }
            if (si > 0 && si < sq) { sq = si; mq = mi; }
        }
        if (mq == -99) {
            x += kx * g.eps; y += ky * g.eps; z += kz * g.eps;
            mr = voronoi_cell_index<double>(g, x, y, z);
            fallbacks++;
            if (mr < 0) done = true;
            continue;
        }
        m = mr; ds = sq;
        x += (sq + g.eps) * kx; y += (sq + g.eps) * ky; z += (sq + g.eps) * kz;
        mr = mq;
        if (mr < 0) done = true;
        return true;
    }
    return false;
}

// FP32: precomputed bisector planes, one 16-byte load per neighbour entry
template<>
SKG_D bool VoronoiStepper<float>::walk(const DevGrid& g, int& m, float& ds) {
    if (qe < 0 && !done) { qb = g.vnoff[mr]; qe = g.vnoff[mr + 1]; }
    while (!done) {
        if (++steps > g.max_steps) { done = true; return false; }
        int qbest = -1;
        const int q0 = qb, q1 = qe;
#if SKG_VOR_NODIV
        // the nearest wall ahead without a division per entry: a candidate s = num/den (den =
        // n.k > 0) is nearer than the best so far when num * bden < bnum * den
        float bnum = 1.f, bden = 0.f;
#pragma unroll 4
        for (int q = q0; q < q1; q++) {
            const float4 pl = __ldg(g.vplane + q);
            const float den = pl.x * kx + pl.y * ky + pl.z * kz;
            const float num = pl.w - (pl.x * x + pl.y * y + pl.z * z);
            if (den > 0.f && num > 0.f && num * bden < bnum * den) { bnum = num; bden = den; qbest = q; }
        }
        scanned += q1 - q0;
        const float sq = (qbest >= 0) ? bnum / bden : FLT_MAX;
#else
        float sq = FLT_MAX;
#pragma unroll 4
        for (int q = q0; q < q1; q++) {
            float4 pl = __ldg(g.vplane + q);
            float ndotk = pl.x * kx + pl.y * ky + pl.z * kz;
            scanned++;
            if (ndotk > 0.f) {
                float si = (pl.w - (pl.x * x + pl.y * y + pl.z * z)) / ndotk;
                if (si > 0.f && si < sq) { sq = si; qbest = q; }
            }
        }
#endif
        if (qbest < 0) {
            x += kx * g.epsf; y += ky * g.epsf; z += kz * g.epsf;
            mr = voronoi_cell_index<float>(g, x, y, z);
            fallbacks++;
            if (mr < 0) done = true;
            else { qb = g.vnoff[mr]; qe = g.vnoff[mr + 1]; }
            continue;
        }
        m = mr;
        x += (sq + g.epsf) * kx; y += (sq + g.epsf) * ky; z += (sq + g.epsf) * kz;
        const int4 e = __ldg(g.vnext + qbest);
        mr = e.x; qb = e.y; qe = e.z;
        if (mr < 0) done = true;
        ds = (mr >= 0) ? sq + g.epsf : sq;   // the nudge is credited to this segment (exact total length)
        return true;
    }
    return false;
}

}  // namespace skg
