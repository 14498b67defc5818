// Stand-in for the reference's DustDistribution (TEST INFRASTRUCTURE): the calls the tree grid's
// set-up makes, declared for the compiled code; the glue drives the grids without that set-up.
#pragma once
#include "Position.hpp"
#include "SimulationItem.hpp"
class DustDistribution : public SimulationItem {
public:
    template<class T> T* interface() { return nullptr; }
    double mass() const { return 0.0; }
    double density(Position) const { return 0.0; }
};
