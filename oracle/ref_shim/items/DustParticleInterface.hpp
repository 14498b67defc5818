// Stand-in for the reference's DustParticleInterface (TEST INFRASTRUCTURE): particles as the
// Voronoi mesh's constructor from an interface reads them.
#pragma once
#include "Vec.hpp"
class DustParticleInterface {
public:
    virtual ~DustParticleInterface() {}
    virtual int numParticles() const = 0;
    virtual Vec particleCenter(int index) const = 0;
};
