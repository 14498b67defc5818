// Stand-in for the reference's ParallelFactory (TEST INFRASTRUCTURE).
#pragma once
#include "Parallel.hpp"
#include "SimulationItem.hpp"
class ParallelFactory : public SimulationItem {
public:
    Parallel* parallel(int = 0) { static Parallel p; return &p; }
};
