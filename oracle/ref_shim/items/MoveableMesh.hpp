// Stand-in for the reference's MoveableMesh (TEST INFRASTRUCTURE); the glue sets the grid's plane
// arrays directly instead of deriving them from meshes.
#pragma once
#include "Array.hpp"
#include "SimulationItem.hpp"
class MoveableMesh : public SimulationItem {
public:
    int numBins() const { return 0; }
    Array mesh() const { return Array(); }
};
