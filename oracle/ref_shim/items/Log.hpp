// Stand-in for the reference's Log (TEST INFRASTRUCTURE): messages are dropped.
#pragma once
#include "SimulationItem.hpp"
class Log : public SimulationItem {
public:
    void info(QString) const {}
    void warning(QString) const {}
    void error(QString) const {}
    void success(QString) const {}
};
