// Stand-in for the reference's SimulationItem (TEST INFRASTRUCTURE): an item of the simulation
// hierarchy without Qt's object tree.  The glue sets the members of the grids it drives directly,
// so find<T>() finds nothing and set-up hooks do nothing.
#pragma once
#include <typeinfo>
#include "QList"
#include "QtLite.hpp"
class SimulationItem {
public:
    virtual ~SimulationItem() {}
    template<class T> T* find(bool = true) const { return nullptr; }
    void setParent(SimulationItem*) {}
    virtual QList<SimulationItem*> interfaceCandidates(const std::type_info&) { QList<SimulationItem*> l; l << this; return l; }
protected:
    virtual void setupSelfBefore() {}
    virtual void setupSelfAfter() {}
};
