// Stand-in for the reference's BoxDustGrid (TEST INFRASTRUCTURE): a dust grid that is also its
// bounding Box; the glue sets the box members directly.
#pragma once
#include "Array.hpp"
#include "DustGrid.hpp"
class BoxDustGrid : public DustGrid, public Box {
protected:
    BoxDustGrid() {}
    void setupSelfBefore() {}
    void setupSelfAfter() {}
public:
    int dimension() const { return 3; }
    Box boundingbox() const { return extent(); }
};
