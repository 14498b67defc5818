// Stand-in for the reference's DustGrid base class (TEST INFRASTRUCTURE): the virtual interface a
// grid implements (DustGrid.hpp:67-124 of the reference), with empty defaults.
#pragma once
#include "Box.hpp"
#include "Position.hpp"
#include "SimulationItem.hpp"
class DustGridPath;
class DustGridPlotFile;
class DustGrid : public SimulationItem {
public:
    bool writeGrid() const { return false; }
    virtual int dimension() const { return 3; }
    virtual int numCells() const { return 0; }
    virtual Box boundingbox() const { return Box(); }
    virtual double weight(int) const { return 1.0; }
    virtual double volume(int) const { return 0.0; }
    virtual int whichcell(Position) const { return -1; }
    virtual Position centralPositionInCell(int) const { return Position(); }
    virtual Position randomPositionInCell(int) const { return Position(); }
    virtual void path(DustGridPath*) const {}
    virtual void write_xy(DustGridPlotFile*) const {}
    virtual void write_xz(DustGridPlotFile*) const {}
    virtual void write_yz(DustGridPlotFile*) const {}
    virtual void write_xyz(DustGridPlotFile*) const {}
};
