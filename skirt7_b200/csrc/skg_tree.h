// skg_tree.h -- host-side octree / k-d tree topology (node boxes, father/child links, cell
// numbers and per-wall neighbour lists) and its flat arrays for the device.
#pragma once
#include "../../include/skirt_b200.h"
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

}  // namespace skg

struct skg_tree {
    skg::Tree t;
};
