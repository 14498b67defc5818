// Stand-in for the reference's PeerToPeerCommunicator (TEST INFRASTRUCTURE): one process.
#pragma once
#include "SimulationItem.hpp"
class PeerToPeerCommunicator : public SimulationItem {
public:
    bool isMultiProc() const { return false; }
    int rank() const { return 0; }
    int size() const { return 1; }
};
