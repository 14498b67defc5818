// ref_grid_glue.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference's own grid traversals, compiled unmodified from its sources (oracle/Makefile
// stages them beside the Qt-lite shims of oracle/ref_shim: the grid classes derive from the
// reference's Qt simulation items, whose headers the shims stand in for):
//   - CartesianDustGrid::path (CartesianDustGrid.cpp:136-283), on a grid whose planes and box this
//     glue sets directly (the reference derives them from its meshes in setupSelfAfter);
//   - VoronoiMesh::path (VoronoiMesh.cpp:778-873) on the mesh VoronoiMesh builds itself from the
//     generator points (VoronoiMesh.cpp:297-420: Voro++, the block lists and the per-block kd-trees
//     of its cell search).
//   - TreeDustGrid::path (TreeDustGrid.cpp:371-643) with its three search methods, on an octree
//     (OctTreeDustGrid) or a k-d tree with alternating directions (BinTreeDustGrid) whose nodes
//     the reference's own node classes create from given split decisions, numbered and linked as
//     TreeDustGrid::setupSelfBefore does (TreeDustGrid.cpp:80-162).
// The tests compare the oracle's restated walks (oracle/oracle.cpp) with these, ray by ray.

#define private public
#define protected public
#include "CartesianDustGrid.hpp"
#include "OctTreeDustGrid.hpp"
#include "BinTreeDustGrid.hpp"
#include "TreeNode.hpp"
#undef private
#undef protected
#include "BinTreeNode.hpp"
#include "DustGridPath.hpp"
#include "OctTreeNode.hpp"
#include "VoronoiMesh.hpp"

#include <cstdint>
#include <vector>

namespace {

// DustGrid::path for n rays; segments of ray i at offsets[i]..offsets[i+1]-1; returns the total
template<class G>
int64_t trace(const G& grid, const double* r, const double* k, int64_t n, int32_t* cells, double* ds,
              int64_t* offsets, int64_t capacity) {
    int64_t pos = 0;
    for (int64_t i = 0; i < n; i++) {
        DustGridPath p(Position(r[3 * i], r[3 * i + 1], r[3 * i + 2]), Direction(k[3 * i], k[3 * i + 1], k[3 * i + 2]));
        grid.path(&p);
        offsets[i] = pos;
        for (int s = 0; s < p.size(); s++) {
            if (pos < capacity) { cells[pos] = p.m(s); ds[pos] = p.ds(s); }
            pos++;
        }
    }
    offsets[n] = pos;
    return pos;
}

}  // namespace

extern "C" {

// CartesianDustGrid with planes xv[nx+1], yv[ny+1], zv[nz+1] and the box ext (xmin, ymin, zmin,
// xmax, ymax, zmax).
int64_t ref_cartesian_paths(const double* ext, const double* xv, int nx, const double* yv, int ny, const double* zv,
                            int nz, const double* r, const double* k, int64_t n, int32_t* cells, double* ds,
                            int64_t* offsets, int64_t capacity) {
    CartesianDustGrid g;
    g._Nx = nx; g._Ny = ny; g._Nz = nz;
    g._xv.resize(nx + 1); g._yv.resize(ny + 1); g._zv.resize(nz + 1);
    for (int i = 0; i <= nx; i++) g._xv[i] = xv[i];
    for (int j = 0; j <= ny; j++) g._yv[j] = yv[j];
    for (int l = 0; l <= nz; l++) g._zv[l] = zv[l];
    g._xmin = ext[0]; g._ymin = ext[1]; g._zmin = ext[2];
    g._xmax = ext[3]; g._ymax = ext[4]; g._zmax = ext[5];
    return trace(g, r, k, n, cells, ds, offsets, capacity);
}

// A tree grid (type 1 octree, 2 k-d tree) over the box ext whose node l is subdivided when
// split[l] != 0 (nodes in creation order), searched with method 0 TopDown, 1 Neighbor, 2 Bookkeeping.
int64_t ref_tree_paths(int type, const double* ext, const uint8_t* split, int64_t nsplit, int search,
                       const double* r, const double* k, int64_t n, int32_t* cells, double* ds, int64_t* offsets,
                       int64_t capacity) {
    TreeDustGrid* g = type == 1 ? static_cast<TreeDustGrid*>(new OctTreeDustGrid())
                                : static_cast<TreeDustGrid*>(new BinTreeDustGrid());
    g->_xmin = ext[0]; g->_ymin = ext[1]; g->_zmin = ext[2];
    g->_xmax = ext[3]; g->_ymax = ext[4]; g->_zmax = ext[5];
    g->_eps = 1e-12 * g->extent().widths().norm();
    g->_search = static_cast<TreeDustGrid::SearchMethod>(search);
    // the nodes: the root of the grid's own kind, children appended in creation order
    g->_tree.push_back(g->createRoot(g->extent()));
    for (size_t l = 0; l < g->_tree.size(); l++) {
        if ((int64_t)l < nsplit && split[l]) {
            TreeNode* node = g->_tree[l];
            node->createchildren(g->_tree.size());
            g->_tree.insert(g->_tree.end(), node->children().begin(), node->children().end());
        }
    }
    g->_Nnodes = g->_tree.size();
    g->_cellnumberv.assign(g->_Nnodes, -1);
    for (int l = 0; l < g->_Nnodes; l++) {
        if (g->_tree[l]->ynchildless()) { g->_cellnumberv[l] = g->_idv.size(); g->_idv.push_back(l); }
    }
    if (g->_search == TreeDustGrid::Neighbor) {
        for (int l = 0; l < g->_Nnodes; l++) g->_tree[l]->addneighbors();
        for (int l = 0; l < g->_Nnodes; l++) g->_tree[l]->sortneighbors();
    }
    const int64_t tot = trace(*g, r, k, n, cells, ds, offsets, capacity);
    delete g;
    return tot;
}

// VoronoiMesh built from nsites generator points in the box ext.
int64_t ref_voronoi_paths(const double* sites, int nsites, const double* ext, const double* r, const double* k,
                          int64_t n, int32_t* cells, double* ds, int64_t* offsets, int64_t capacity) {
    std::vector<Vec> particles(nsites);
    for (int m = 0; m < nsites; m++) particles[m] = Vec(sites[3 * m], sites[3 * m + 1], sites[3 * m + 2]);
    VoronoiMesh mesh(particles, Box(ext[0], ext[1], ext[2], ext[3], ext[4], ext[5]), nullptr);
    return trace(mesh, r, k, n, cells, ds, offsets, capacity);
}

}  // extern "C"
