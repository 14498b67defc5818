// Stand-in for the reference's DustGridPlotFile (TEST INFRASTRUCTURE): grid plots are not written.
#pragma once
#include "QtLite.hpp"
class DustGridPlotFile {
public:
    void writeLine(double, double, double, double) {}
    void writeLine(double, double, double, double, double, double) {}
    void writeRectangle(double, double, double, double) {}
    void writeCube(double, double, double, double, double, double) {}
};
