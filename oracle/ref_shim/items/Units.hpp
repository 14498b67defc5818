// Stand-in for the reference's Units (TEST INFRASTRUCTURE): the V-band extinction coefficient the
// tree node calculators use (Units::kappaV, Units.cpp:29 of the reference: 2600 m2/kg).
#pragma once
#include "SimulationItem.hpp"
class Units : public SimulationItem {
public:
    static double kappaV() { return 2600.; }
};
