// ref_glue.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Exposes the reference's own compiled classes (built in place from the SKIRT7 sources by
// oracle/Makefile into oracle/_ref/libskirt_ref.so) to the tests, which compare them with the
// oracle's restatement and with the library's host code:
//   - DustGridPath::pathlength and ::moveInside (SKIRTcore/DustGridPath.cpp);
//   - the octree / k-d tree node classes: subdivision, neighbour lists and their order
//     (SKIRTcore/TreeNode.cpp, OctTreeNode.cpp, BinTreeNode.cpp), driven the way
//     TreeDustGrid::setupSelfBefore drives them (TreeDustGrid.cpp:80-162);
//   - SpecialFunctions::LambertW1 and the SersicFunction tables;
//   - Voro++ cell neighbours, volumes, centroids and extents, computed the way
//     VoronoiMesh::buildMesh calls it (VoronoiMesh.cpp:334-390).

// the node classes keep their neighbour lists protected; this test-only glue reads them
#define protected public
#include "TreeNode.hpp"
#include "OctTreeNode.hpp"
#include "BinTreeNode.hpp"
#undef protected
#include "Box.hpp"
#include "DustGridPath.hpp"
#include "FatalError.hpp"
#include "container.hh"
#include "SersicFunction.hpp"
#include "SpecialFunctions.hpp"

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

FatalError::FatalError(QString message, const char*, int, const char*) { _message.push_back(message); }
QStringList FatalError::message() const { return _message; }

extern "C" {

// DustGridPath built from segment lengths ds[] in cells 0..n-1 with kappa*rho kr[] per cell;
// returns pathlength(tau).
double ref_pathlength(const double* ds, const double* kr, int n, double tau) {
    DustGridPath p(Position(0, 0, 0), Direction(0, 0, 1));
    for (int i = 0; i < n; i++) p.addSegment(i, ds[i]);
    p.fillOpticalDepth([kr](int m) { return kr[m]; });
    return p.pathlength(tau);
}

// DustGridPath::moveInside; writes the final position and the entry segment lengths; returns the
// number of segments (or -1 for the OUTSIDE position).
int ref_moveinside(const double* box, double eps, const double* r, const double* k, double* out_r, double* seg) {
    DustGridPath p(Position(r[0], r[1], r[2]), Direction(k[0], k[1], k[2]));
    Box b(box[0], box[1], box[2], box[3], box[4], box[5]);
    Position q = p.moveInside(b, eps);
    double x, y, z;
    q.cartesian(x, y, z);
    out_r[0] = x; out_r[1] = y; out_r[2] = z;
    for (int i = 0; i < p.size(); i++) seg[i] = p.ds(i);
    if (std::isinf(x)) return -1;
    return p.size();
}

// Builds a tree with the reference node classes from split decisions in creation order, adds and
// sorts the neighbour lists like TreeDustGrid::setupSelfBefore, and returns the flattened lists
// of every leaf (CSR by 6*node+wall; other nodes get empty lists).  type 1 = octree, 2 = k-d tree
// with alternating directions.  Returns the node count (or -needed if the buffers are too small).
int64_t ref_tree_neighbors(int type, const double* ext, const uint8_t* split, int64_t nsplit,
                           int64_t max_nodes, double* boxes, int64_t* offsets, int32_t* ids, int64_t max_ids) {
    std::vector<TreeNode*> tree;
    Box extent(ext[0], ext[1], ext[2], ext[3], ext[4], ext[5]);
    if (type == 1) tree.push_back(new OctTreeNode(0, 0, extent));
    else tree.push_back(new BinTreeNode(0, 0, extent));
    for (size_t l = 0; l < tree.size(); l++) {
        if ((int64_t)l < nsplit && split[l]) {
            TreeNode* node = tree[l];
            node->createchildren(tree.size());
            tree.insert(tree.end(), node->children().begin(), node->children().end());
        }
    }
    int64_t n = tree.size();
    for (int64_t l = 0; l < n; l++) tree[l]->ensureneighborlists();
    for (int64_t l = 0; l < n; l++) tree[l]->addneighbors();
    for (int64_t l = 0; l < n; l++) tree[l]->sortneighbors();
    if (n > max_nodes) { for (auto t : tree) delete t; return -n; }
    int64_t q = 0;
    offsets[0] = 0;
    for (int64_t l = 0; l < n; l++) {
        TreeNode* node = tree[l];
        boxes[6 * l] = node->xmin(); boxes[6 * l + 1] = node->ymin(); boxes[6 * l + 2] = node->zmin();
        boxes[6 * l + 3] = node->xmax(); boxes[6 * l + 4] = node->ymax(); boxes[6 * l + 5] = node->zmax();
        for (int w = 0; w < 6; w++) {
            if (node->ynchildless()) {
                for (TreeNode* nb : node->_neighbors[w]) {
                    if (q < max_ids) ids[q] = nb->id();
                    q++;
                }
            }
            offsets[6 * l + w + 1] = q;
        }
    }
    for (auto t : tree) delete t;
    return q > max_ids ? -q : n;
}

// Voro++ tessellation of n sites clipped to the extent with nb^3 blocks (VoronoiMesh.cpp:334-390);
// writes per site its neighbour ids (walls -1..-6), volume, centroid and bounding box.
int64_t ref_voronoi(const double* sites, int n, const double* ext, int nb, int64_t* offsets, int32_t* ids,
                    int64_t max_ids, double* volume, double* centroid, double* bbox) {
    voro::container con(ext[0], ext[3], ext[1], ext[4], ext[2], ext[5], nb, nb, nb, false, false, false, 8);
    for (int m = 0; m < n; m++) con.put(m, sites[3 * m], sites[3 * m + 1], sites[3 * m + 2]);
    std::vector<std::vector<int>> nbrs(n);
    voro::c_loop_all loop(con);
    if (loop.start()) do {
        voro::voronoicell_neighbor cell;
        if (!con.compute_cell(cell, loop)) return -1;
        int m = loop.pid();
        double x, y, z;
        loop.pos(x, y, z);
        double cx, cy, cz;
        cell.centroid(cx, cy, cz);
        centroid[3 * m] = cx + x; centroid[3 * m + 1] = cy + y; centroid[3 * m + 2] = cz + z;
        volume[m] = cell.volume();
        std::vector<double> v;
        cell.vertices(x, y, z, v);
        double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
        for (size_t i = 0; i < v.size(); i += 3)
            for (int c = 0; c < 3; c++) { lo[c] = std::min(lo[c], v[i + c]); hi[c] = std::max(hi[c], v[i + c]); }
        for (int c = 0; c < 3; c++) { bbox[6 * m + c] = lo[c]; bbox[6 * m + 3 + c] = hi[c]; }
        cell.neighbors(nbrs[m]);
    } while (loop.inc());
    int64_t q = 0;
    offsets[0] = 0;
    for (int m = 0; m < n; m++) {
        for (int id : nbrs[m]) { if (q < max_ids) ids[q] = id; q++; }
        offsets[m + 1] = q;
    }
    return q > max_ids ? -q : q;
}

// SpecialFunctions::LambertW1 (SpecialFunctions.cpp:579)
double ref_lambertw1(double z) { return SpecialFunctions::LambertW1(z); }

// SersicFunction(n): the normalised profile, mass and inverse mass at the given points
// (SersicFunction.cpp:17-122)
void ref_sersic(double n, const double* s, int ns, double* S, double* M, const double* X, int nx, double* inv) {
    SersicFunction f(n);
    for (int i = 0; i < ns; i++) { S[i] = f(s[i]); M[i] = f.mass(s[i]); }
    for (int i = 0; i < nx; i++) inv[i] = f.inversemass(X[i]);
}

}  // extern "C"
