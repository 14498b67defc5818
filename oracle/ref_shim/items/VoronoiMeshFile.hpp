// Stand-in for the reference's VoronoiMeshFile (TEST INFRASTRUCTURE): the reader interface the
// Voronoi mesh's file constructor calls; the glue builds meshes from particle vectors instead.
#pragma once
#include "Vec.hpp"
class VoronoiMeshFile {
public:
    virtual ~VoronoiMeshFile() {}
    virtual void open() {}
    virtual bool read() { return false; }
    virtual Vec particle() const { return Vec(); }
    virtual double value(int) const { return 0.0; }
    virtual void close() {}
};
