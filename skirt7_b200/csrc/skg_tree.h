// skg_tree.h -- host-side octree / k-d tree topology (node boxes, father/child links, cell
// numbers and per-wall neighbour lists) and its flat arrays for the device.
#pragma once
#include "../../include/skirt_b200.h"
#include <vector_types.h>
#include <cstdint>
#include <functional>
#include <vector>

namespace skg {

struct TNode {
    double box[6];          // xmin, ymin, zmin, xmax, ymax, zmax
    int father = -1;
    int child = -1;         // id of child 0 (children are consecutive)
    int cell = -1;          // cell number of a leaf
    int level = 0;
    signed char dir = -1;   // split direction of a binary node
};

struct Tree {
    int type = SKG_GRID_OCTREE;
    double ext[6];
    std::vector<TNode> nodes;
    std::vector<std::vector<int>> nbrs;   // [6*l + wall] during construction
    int ncells = 0;

    // flat arrays (after flatten())
    std::vector<double> box;
    std::vector<int32_t> child, father, cell, cell_node;
    std::vector<int8_t> dir;
    std::vector<int64_t> nbroff;
    std::vector<int32_t> nbr;

    void split(int l);
    void make_neighbors(int wall1, int n1, int n2);
    void add_neighbors(int l);
    void sort_neighbors(int l);
    void finish(bool with_neighbors);
    void flatten();
    void fill_grid(skg_grid* g) const;
    void build(int min_level, int max_level, double max_mass_fraction, double max_optical_depth,
               double max_dens_disp, double total_mass,
               const std::function<void(const std::vector<int>&, std::vector<double>&, std::vector<double>&,
                                        std::vector<double>&)>& sample);
    void build_from_splits(const uint8_t* split, int64_t nsplit);
};

// Rope-linked tree for the FP32 production walk (see build_rope_tree in skg_host.cpp).
//   lrec: 4 float4 per leaf, leaves in depth-first order
//     [0] = (xmin, ymin, zmin, density placeholder)   [1] = (xmax, ymax, zmax, int cell number)
//     [2] = int ropes of walls 0..3                   [3] = int ropes of walls 4,5, 0, 0
//   irec: 3 float4 per internal node: (split x, y, z, int split direction or -1 for an octree node),
//         then 8 int child references
//   references: >= 0 leaf index, -1 none (outside the domain), <= -2 internal node -(ref + 2)
//
// Lattice form, for trees whose nodes all split at their midpoints (OctTreeNode, BinTreeNode): a
// node's extent along axis a is the interval of level l_a and index i_a of the root's extent, coded
// as the 21-bit centre c_a = (2 i_a + 1) << (20 - l_a) in units u_a = extent_a / 2^21, so that
// every wall is fmaf(integer, u_a, origin_a) -- the same float on both sides of it.
//   prec: 2 uint4 (32 bytes) per leaf, in cell-number order (leaf reference = cell number)
//     word 0      density (float bits; 0 until embedded)
//     words 1-2   codes: bits 0-20 c_x, 21-41 c_y, 42-62 c_z of the 64-bit word (w2:w1)
//     words 3-7   ropes of walls 0..5, 26 bits each at bit 26*wall of the 160-bit string
//                 (0x3FFFFFF none, < 2^25 cell number, else internal node + 2^25)
//   irec as above, with leaf references replaced by cell numbers and split points computed as
//   fmaf(c, u, origin) from the node's centre codes.
struct RopeTree {
    std::vector<float4> lrec, irec;
    std::vector<int> cell_leaf;
    int root_ref = -1;
    bool lattice = false;
    std::vector<uint4> prec;
    float lorg[3] = {0, 0, 0}, lunit[3] = {0, 0, 0};
};
// Builds the lattice form when every node fits the lattice (and allow_lattice), else the 64-byte
// leaf records.
void build_rope_tree(const skg_grid& g, RopeTree& out, bool allow_lattice = true);

}  // namespace skg

struct skg_tree {
    skg::Tree t;
};
