// Stand-in for the reference's Random (TEST INFRASTRUCTURE): declared for the grid code that samples
// positions in cells, which the glue does not call.
#pragma once
#include "Array.hpp"
#include "Box.hpp"
#include "Position.hpp"
#include "SimulationItem.hpp"
class Random : public SimulationItem {
public:
    double uniform() { return 0.5; }
    Position position(const Box& box) { return Position(box.center()); }
};
