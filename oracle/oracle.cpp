// oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement (FP64, scalar per thread) of SKIRT7's photon-packet life cycle, used as the
// parity checker for the CUDA path and as the timed CPU baseline.  Only tests/, the smoke check
// and the CPU-baseline leg of bench.py may load it; the product never does.
//
// Every function cites the reference lines it restates (paths relative to the SKIRT7 tree).
// Arithmetic order follows the reference so that traversals are bit-identical to it; compile
// with -ffp-contract=off (the reference's x86-64 build has no FMA contraction).
//
// Parity is pinned by (a) the reference's own translation units compiled from its sources into
// oracle/_ref (DustGridPath::pathlength/moveInside, the tree node classes' neighbour lists) and
// compared against this restatement in tests/test_oracle_pins.py, and (b) the reference's
// built-in self-checks (face-on optical depth, energy conservation, transparent flux).

#include "../include/skirt_b200.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace orc {

using std::vector;

static thread_local std::string g_err;

// ---------------------------------------------------------------------------------------------
// Vec / Box (Fundamentals/Vec.hpp, Fundamentals/Box.hpp)

struct Vec {
    double x, y, z;
    Vec() : x(0), y(0), z(0) {}
    Vec(double a, double b, double c) : x(a), y(b), z(c) {}
    double norm2() const { return x*x + y*y + z*z; }
    double norm() const { return std::sqrt(x*x + y*y + z*z); }
};
static inline Vec operator+(Vec a, Vec b) { return Vec(a.x+b.x, a.y+b.y, a.z+b.z); }
static inline Vec operator-(Vec a, Vec b) { return Vec(a.x-b.x, a.y-b.y, a.z-b.z); }
static inline Vec operator*(double s, Vec b) { return Vec(s*b.x, s*b.y, s*b.z); }
static inline Vec operator*(Vec b, double s) { return Vec(b.x*s, b.y*s, b.z*s); }
static inline double dot(Vec a, Vec b) { return a.x*b.x + a.y*b.y + a.z*b.z; }

struct Box {
    double xmin, ymin, zmin, xmax, ymax, zmax;
    bool contains(Vec r) const {  // Box.hpp:80-81
        return r.x >= xmin && r.x <= xmax && r.y >= ymin && r.y <= ymax && r.z >= zmin && r.z <= zmax;
    }
    double volume() const { return (xmax-xmin) * (ymax-ymin) * (zmax-zmin); }
    Vec fracpos(double a, double b, double c) const {  // Box.hpp:105-106
        return Vec(xmin + a*(xmax-xmin), ymin + b*(ymax-ymin), zmin + c*(zmax-zmin));
    }
    void cellindices(int& i, int& j, int& k, Vec r, int nx, int ny, int nz) const {  // Box.hpp:120-125
        i = std::max(0, std::min(nx-1, static_cast<int>(nx*(r.x-xmin)/(xmax-xmin))));
        j = std::max(0, std::min(ny-1, static_cast<int>(ny*(r.y-ymin)/(ymax-ymin))));
        k = std::max(0, std::min(nz-1, static_cast<int>(nz*(r.z-zmin)/(zmax-zmin))));
    }
};

// ---------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11), the counter-based generator of the library's
// device kernels, restated for the checks that need the device's samples (tree node masses) or
// streams keyed by packet (packet-range runs): key = seed, counter words = (block, node id lo, node id hi,
// stream), deviates ((u32 + 0.5) * 2^-32).
struct Philox {
    uint32_t k0 = 0, k1 = 0, c1 = 0, c2 = 0, c3 = 0, c0 = 0, b[4] = {0, 0, 0, 0}; int left = 0;
    Philox() = default;
    Philox(uint64_t seed, uint64_t id, uint32_t stream)
        : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), c1((uint32_t)id), c2((uint32_t)(id >> 32)), c3(stream) {}
    double uniform() {
        if (left == 0) {
            uint32_t x0 = c0, x1 = c1, x2 = c2, x3 = c3, a = k0, bb = k1;
            for (int r = 0; r < 10; r++) {
                uint64_t p0 = (uint64_t)0xD2511F53u * x0, p1 = (uint64_t)0xCD9E8D57u * x2;
                uint32_t y0 = (uint32_t)(p1 >> 32) ^ x1 ^ a, y1 = (uint32_t)p1;
                uint32_t y2 = (uint32_t)(p0 >> 32) ^ x3 ^ bb, y3 = (uint32_t)p0;
                x0 = y0; x1 = y1; x2 = y2; x3 = y3;
                a += 0x9E3779B9u; bb += 0xBB67AE85u;
            }
            b[0] = x0; b[1] = x1; b[2] = x2; b[3] = x3; left = 4; c0++;
        }
        return ((double)b[4 - (left--)] + 0.5) * 2.3283064365386963e-10;
    }
};

// ---------------------------------------------------------------------------------------------
// Random (SKIRTcore/Random.cpp): one MT19937 state per thread, seeded seed+thread (:41-56),
// uniform deviates excluding 0 and 1 (:90-127).

struct Rng {
    unsigned long mt[624];
    int mti;
    // packet-range runs draw from a counter-based stream keyed by the packet instead of the
    // thread's MT19937 stream (orc_simulate_packets)
    bool counter = false;
    Philox ph;
    void init(unsigned long seed) {            // Random.cpp:46-50
        mt[0] = seed & 0xffffffffUL;
        for (mti = 1; mti < 624; mti++) mt[mti] = (69069UL * mt[mti-1]) & 0xffffffffUL;
    }
    double uniform() {                          // Random.cpp:90-127
        if (counter) return ph.uniform();
        static const unsigned long mag01[2] = {0x0UL, 0x9908b0dfUL};
        double ans;
        do {
            unsigned long y;
            if (mti >= 624) {
                int kk;
                for (kk = 0; kk < 227; kk++) {
                    y = (mt[kk] & 0x80000000UL) | (mt[kk+1] & 0x7fffffffUL);
                    mt[kk] = mt[kk+397] ^ (y >> 1) ^ mag01[y & 0x1UL];
                }
                for (; kk < 623; kk++) {
                    y = (mt[kk] & 0x80000000UL) | (mt[kk+1] & 0x7fffffffUL);
                    mt[kk] = mt[kk-227] ^ (y >> 1) ^ mag01[y & 0x1UL];
                }
                y = (mt[623] & 0x80000000UL) | (mt[0] & 0x7fffffffUL);
                mt[623] = mt[396] ^ (y >> 1) ^ mag01[y & 0x1UL];
                mti = 0;
            }
            y = mt[mti++];
            y ^= (y >> 11);
            y ^= (y << 7) & 0x9d2c5680UL;
            y ^= (y << 15) & 0xefc60000UL;
            y ^= (y >> 18);
            ans = static_cast<double>(y) / static_cast<unsigned long>(0xffffffffUL);
        } while (ans <= 0.0 || ans >= 1.0);
        return ans;
    }
    double exponcutoff(double xmax) {           // Random.cpp:163-176
        if (xmax == 0.0) return 0.0;
        else if (xmax < 1e-10) return uniform()*xmax;
        double x = -std::log(1.0 - uniform()*(1.0 - std::exp(-xmax)));
        while (x > xmax) x = -std::log(1.0 - uniform()*(1.0 - std::exp(-xmax)));
        return x;
    }
    Vec direction() {                           // Random.cpp:180-185 + Direction.cpp:12-38
        double theta = std::acos(2.0*uniform() - 1.0);
        double phi = 2.0*M_PI*uniform();
        return dirFromAngles(theta, phi);
    }
    static Vec dirFromAngles(double theta, double phi) {   // Direction.cpp:12-38
        const double eps = 1e-8;
        if (theta <= eps) return Vec(0, 0, 1);
        if (theta >= M_PI-eps) return Vec(0, 0, -1);
        double st = std::sin(theta);
        return Vec(st*std::cos(phi), st*std::sin(phi), std::cos(theta));
    }
    Vec direction(Vec k, double costheta) {     // Random.cpp:189-223
        double phi = 2.0*M_PI*uniform();
        double cosphi = std::cos(phi), sinphi = std::sin(phi);
        double sintheta = std::sqrt(std::fabs((1.0-costheta)*(1.0+costheta)));
        double kx = k.x, ky = k.y, kz = k.z;
        if (kz > 0.99999) return Vec(cosphi*sintheta, sinphi*sintheta, costheta);
        if (kz < -0.99999) return Vec(cosphi*sintheta, sinphi*sintheta, -costheta);
        double root = std::sqrt((1.0-kz)*(1.0+kz));
        return Vec(sintheta/root*(-kx*kz*cosphi + ky*sinphi) + kx*costheta,
                   -sintheta/root*(ky*kz*cosphi + kx*sinphi) + ky*costheta,
                   root*sintheta*cosphi + kz*costheta);
    }
    Vec position(const Box& b) {                // Random.cpp:227-235
        double x = uniform(); double y = uniform(); double z = uniform();
        return b.fracpos(x, y, z);
    }
};

// ---------------------------------------------------------------------------------------------
// NR helpers (Fundamentals/NR.hpp)

static inline int locate_basic(const double* xv, double x, int n) {     // NR.hpp:114-127
    int jl = -1, ju = n;
    while (ju-jl > 1) { int jm = (ju+jl) >> 1; if (x < xv[jm]) ju = jm; else jl = jm; }
    return jl;
}
static inline int locate_clip(const double* xv, int size, double x) {   // NR.hpp:145-151
    if (x < xv[0]) return 0;
    return locate_basic(xv, x, size-1);
}
static inline int locate_fail(const double* xv, int size, double x) {   // NR.hpp:155-160
    if (x > xv[size-1]) return -1;
    return locate_basic(xv, x, size-1);
}
static inline double interpolate_linlin(double x, double x1, double x2, double f1, double f2) {  // NR.hpp:296-299
    return f1 + ((x-x1)/(x2-x1))*(f2-f1);
}
static inline double interpolate_loglog(double x, double x1, double x2, double f1, double f2) { // NR.hpp:318-345
    x = std::log10(x); x1 = std::log10(x1); x2 = std::log10(x2);
    bool logf = f1 > 0 && f2 > 0;
    if (logf) { f1 = std::log10(f1); f2 = std::log10(f2); }
    double fx = f1 + ((x-x1)/(x2-x1))*(f2-f1);
    if (logf) fx = std::pow(10, fx);
    return fx;
}
static void cdf(vector<double>& Pv, const vector<double>& pv) {           // NR.hpp:388-394
    int n = pv.size();
    Pv.assign(n+1, 0.0);
    for (int i = 0; i < n; i++) Pv[i+1] = Pv[i] + pv[i];
    double t = Pv[n];
    for (auto& p : Pv) p /= t;
}

// ---------------------------------------------------------------------------------------------
// DustGridPath (SKIRTcore/DustGridPath.hpp/.cpp)

struct Segment { int m; double ds, s, dtau, tau; };

struct Path {
    Vec r, k;
    double s = 0;
    vector<Segment> v;
    Path() { v.reserve(1000); }                               // DustGridPath.cpp:17-26
    void clear() { s = 0; v.clear(); }                        // :38-42
    void addSegment(int m, double ds) {                       // :46-53
        if (ds > 0) { s += ds; v.push_back(Segment{m, ds, s, 0, 0}); }
    }
    bool moveInside(const Box& box, double eps, Vec& out) {   // :57-150 (false = OUTSIDE)
        double kx = k.x, ky = k.y, kz = k.z;
        double rx = r.x, ry = r.y, rz = r.z;
        if (rx <= box.xmin) {
            if (kx <= 0.0) return false;
            double ds = (box.xmin-rx)/kx; addSegment(-1, ds);
            rx = box.xmin + eps; ry += ky*ds; rz += kz*ds;
        } else if (rx >= box.xmax) {
            if (kx >= 0.0) return false;
            double ds = (box.xmax-rx)/kx; addSegment(-1, ds);
            rx = box.xmax - eps; ry += ky*ds; rz += kz*ds;
        }
        if (ry <= box.ymin) {
            if (ky <= 0.0) return false;
            double ds = (box.ymin-ry)/ky; addSegment(-1, ds);
            rx += kx*ds; ry = box.ymin + eps; rz += kz*ds;
        } else if (ry >= box.ymax) {
            if (ky >= 0.0) return false;
            double ds = (box.ymax-ry)/ky; addSegment(-1, ds);
            rx += kx*ds; ry = box.ymax - eps; rz += kz*ds;
        }
        if (rz <= box.zmin) {
            if (kz <= 0.0) return false;
            double ds = (box.zmin-rz)/kz; addSegment(-1, ds);
            rx += kx*ds; ry += ky*ds; rz = box.zmin + eps;
        } else if (rz >= box.zmax) {
            if (kz >= 0.0) return false;
            double ds = (box.zmax-rz)/kz; addSegment(-1, ds);
            rx += kx*ds; ry += ky*ds; rz = box.zmax - eps;
        }
        out = Vec(rx, ry, rz);
        return true;
    }
    template<typename F> void fillOpticalDepth(F kapparho) {  // DustGridPath.hpp:117-129
        double tau = 0;
        for (auto& sg : v) { double dtau = kapparho(sg.m)*sg.ds; tau += dtau; sg.dtau = dtau; sg.tau = tau; }
    }
    template<typename F> double opticalDepth(F kapparho, double distance = DBL_MAX) const {  // :97-108
        double tau = 0;
        for (const auto& sg : v) { tau += kapparho(sg.m)*sg.ds; if (sg.s > distance) break; }
        return tau;
    }
    double tau() const { return v.empty() ? 0 : v.back().tau; }   // DustGridPath.cpp:154-158
    double pathlength(double tau) const {                          // DustGridPath.cpp:162-173
        int N = v.size();
        if (N > 0 && tau > 0) {
            // NR::locate<Segment> on cumulative tau (NR.hpp:76-95)
            int i;
            if (tau < v[0].tau) i = -1;
            else if (v[N-1].tau < tau) i = N-1;
            else {
                int jl = -1, ju = N;
                while (ju-jl > 1) { int jm = (ju+jl) >> 1; if (tau < v[jm].tau) ju = jm; else jl = jm; }
                if (jl <= 0) i = 0; else if (jl >= N-2) i = N-2; else i = jl;
            }
            if (i < 0) return interpolate_linlin(tau, 0, v[0].tau, 0, v[0].s);
            if (i < N-1) return interpolate_linlin(tau, v[i].tau, v[i+1].tau, v[i].s, v[i+1].s);
            return v[N-1].s;
        }
        return 0;
    }
};

// ---------------------------------------------------------------------------------------------
// Dust grids

struct Grid {
    Box ext;
    int ncells = 0;
    virtual ~Grid() {}
    virtual void path(Path& p, long* fallbacks) const = 0;       // DustGrid::path (DustGrid.hpp:106)
    virtual int whichcell(Vec r) const = 0;                       // DustGrid::whichcell (:89)
    virtual Vec randomPositionInCell(int m, Rng& rng) const = 0;  // DustGrid::randomPositionInCell (:97)
    virtual double volume(int m) const = 0;
};

// CartesianDustGrid (SKIRTcore/CartesianDustGrid.cpp)
struct CartesianGrid : Grid {
    int Nx, Ny, Nz;
    vector<double> xv, yv, zv;
    int index(int i, int j, int k) const { return k + Nz*j + Nz*Ny*i; }   // :326-329
    Box box(int m) const {                                                  // :333-343
        int i = m/(Nz*Ny), j = (m/Nz) % Ny, k = m % Nz;
        return Box{xv[i], yv[j], zv[k], xv[i+1], yv[j+1], zv[k+1]};
    }
    double volume(int m) const override { return box(m).volume(); }        // :104-107
    int whichcell(Vec r) const override {                                   // :109-118
        int i = locate_fail(xv.data(), Nx+1, r.x);
        int j = locate_fail(yv.data(), Ny+1, r.y);
        int k = locate_fail(zv.data(), Nz+1, r.z);
        if (i < 0 || j < 0 || k < 0) return -1;
        return index(i, j, k);
    }
    Vec randomPositionInCell(int m, Rng& rng) const override { return rng.position(box(m)); }
    void path(Path& p, long*) const override {                              // :136-283
        p.clear();
        double kx = p.k.x, ky = p.k.y, kz = p.k.z;
        double x = p.r.x, y = p.r.y, z = p.r.z;
        double ds, dsx, dsy, dsz;
        const double xmin = ext.xmin, xmax = ext.xmax, ymin = ext.ymin, ymax = ext.ymax,
                     zmin = ext.zmin, zmax = ext.zmax;
        if (x < xmin) {
            if (kx <= 0.0) return p.clear();
            ds = (xmin-x)/kx; p.addSegment(-1, ds);
            x = xmin + 1e-8*(xv[1]-xv[0]); y += ky*ds; z += kz*ds;
        } else if (x > xmax) {
            if (kx >= 0.0) return p.clear();
            ds = (xmax-x)/kx; p.addSegment(-1, ds);
            x = xmax - 1e-8*(xv[Nx]-xv[Nx-1]); y += ky*ds; z += kz*ds;
        }
        if (y < ymin) {
            if (ky <= 0.0) return p.clear();
            ds = (ymin-y)/ky; p.addSegment(-1, ds);
            x += kx*ds; y = ymin + 1e-8*(yv[1]-yv[0]); z += kz*ds;
        } else if (y > ymax) {
            if (ky >= 0.0) return p.clear();
            ds = (ymax-y)/ky; p.addSegment(-1, ds);
            x += kx*ds; y = ymax - 1e-8*(yv[Ny]-yv[Ny-1]); z += kz*ds;
        }
        if (z < zmin) {
            if (kz <= 0.0) return p.clear();
            ds = (zmin-z)/kz; p.addSegment(-1, ds);
            x += kx*ds; y += ky*ds; z = zmin + 1e-8*(zv[1]-zv[0]);
        } else if (z > zmax) {
            if (kz >= 0.0) return p.clear();
            ds = (zmax-z)/kz; p.addSegment(-1, ds);
            x += kx*ds; y += ky*ds; z = zmax - 1e-8*(zv[Nz]-zv[Nz-1]);
        }
        if (x < xmin || x > xmax || y < ymin || y > ymax || z < zmin || z > zmax) return p.clear();
        int i = locate_clip(xv.data(), Nx+1, x);
        int j = locate_clip(yv.data(), Ny+1, y);
        int k = locate_clip(zv.data(), Nz+1, z);
        long guard = 0;
        while (true) {
            if (++guard > (1L << 22)) return;   // test guard
            int m = index(i, j, k);
            double xE = (kx < 0.0) ? xv[i] : xv[i+1];
            double yE = (ky < 0.0) ? yv[j] : yv[j+1];
            double zE = (kz < 0.0) ? zv[k] : zv[k+1];
            dsx = (std::fabs(kx) > 1e-15) ? (xE-x)/kx : DBL_MAX;
            dsy = (std::fabs(ky) > 1e-15) ? (yE-y)/ky : DBL_MAX;
            dsz = (std::fabs(kz) > 1e-15) ? (zE-z)/kz : DBL_MAX;
            if (dsx <= dsy && dsx <= dsz) {
                ds = dsx; p.addSegment(m, ds);
                i += (kx < 0.0) ? -1 : 1;
                if (i >= Nx || i < 0) return;
                x = xE; y += ky*ds; z += kz*ds;
            } else if (dsy < dsx && dsy <= dsz) {
                ds = dsy; p.addSegment(m, ds);
                j += (ky < 0.0) ? -1 : 1;
                if (j >= Ny || j < 0) return;
                x += kx*ds; y = yE; z += kz*ds;
            } else if (dsz < dsx && dsz < dsy) {
                ds = dsz; p.addSegment(m, ds);
                k += (kz < 0.0) ? -1 : 1;
                if (k >= Nz || k < 0) return;
                x += kx*ds; y += ky*ds; z = zE;
            } else {
                return;  // unreachable for finite ds; guards NaN directions (the reference would spin)
            }
        }
    }
};

// TreeDustGrid over flat arrays (SKIRTcore/TreeDustGrid.cpp, TreeNode.cpp, OctTreeNode.cpp,
// BinTreeNode.cpp).  Node l: box, first child id (children consecutive), father, split dir.
struct TreeGrid : Grid {
    int nnodes;
    vector<Box> box;
    vector<int> child, father, cell;
    vector<signed char> dir;
    vector<int64_t> nbroff;
    vector<int> nbr;
    vector<int> idv;          // leaf node id for each cell (TreeDustGrid.cpp:106-116)
    int search;
    double eps;

    double volume(int m) const override { return box[idv[m]].volume(); }    // :332-338
    Vec randomPositionInCell(int m, Rng& rng) const override { return rng.position(box[idv[m]]); }
    int childOf(int l, Vec r) const {
        int c0 = child[l];
        if (dir[l] < 0) {                                   // OctTreeNode::child (OctTreeNode.cpp:184-189)
            const Box& b = box[c0];
            int o = (r.x < b.xmax ? 0 : 1) + (r.y < b.ymax ? 0 : 2) + (r.z < b.zmax ? 0 : 4);
            return c0 + o;
        }
        const Box& b = box[c0];                             // BinTreeNode::child (BinTreeNode.cpp:326-335)
        switch (dir[l]) {
            case 0: return r.x < b.xmax ? c0 : c0+1;
            case 1: return r.y < b.ymax ? c0 : c0+1;
            default: return r.z < b.zmax ? c0 : c0+1;
        }
    }
    int whichnode(int l, Vec r) const {                     // TreeNode::whichnode (TreeNode.cpp:70-80)
        if (!box[l].contains(r)) return -1;
        while (child[l] >= 0) l = childOf(l, r);
        return l;
    }
    int whichnode(int l, int wall, Vec r) const {           // TreeNode::whichnode(wall) (:84-93)
        for (int64_t q = nbroff[6*l+wall]; q < nbroff[6*l+wall+1]; q++)
            if (box[nbr[q]].contains(r)) return nbr[q];
        return -1;
    }
    int whichcell(Vec r) const override {                   // TreeDustGrid.cpp:349-353
        int l = whichnode(0, r);
        return l >= 0 ? cell[l] : -1;
    }
    void path(Path& p, long* fallbacks) const override {    // TreeDustGrid.cpp:371-643
        p.clear();
        Vec bfr;
        if (!p.moveInside(ext, eps, bfr)) bfr = Vec(INFINITY, INFINITY, INFINITY);
        int node = whichnode(0, bfr);
        if (node < 0) return p.clear();
        double x = bfr.x, y = bfr.y, z = bfr.z;
        double kx = p.k.x, ky = p.k.y, kz = p.k.z;
        long guard = 0;
        if (search == SKG_SEARCH_TOPDOWN || search == SKG_SEARCH_NEIGHBOR) {
            while (node >= 0) {
                if (++guard > (1L << 22)) break;   // test guard
                const Box& b = box[node];
                double xnext = (kx < 0.0) ? b.xmin : b.xmax;
                double ynext = (ky < 0.0) ? b.ymin : b.ymax;
                double znext = (kz < 0.0) ? b.zmin : b.zmax;
                double dsx = (std::fabs(kx) > 1e-15) ? (xnext-x)/kx : DBL_MAX;
                double dsy = (std::fabs(ky) > 1e-15) ? (ynext-y)/ky : DBL_MAX;
                double dsz = (std::fabs(kz) > 1e-15) ? (znext-z)/kz : DBL_MAX;
                double ds; int wall;
                if (dsx <= dsy && dsx <= dsz) { ds = dsx; wall = (kx < 0.0) ? 0 : 1; }
                else if (dsy <= dsx && dsy <= dsz) { ds = dsy; wall = (ky < 0.0) ? 2 : 3; }
                else { ds = dsz; wall = (kz < 0.0) ? 4 : 5; }
                p.addSegment(cell[node], ds);
                x += (ds+eps)*kx; y += (ds+eps)*ky; z += (ds+eps)*kz;
                int oldnode = node;
                if (search == SKG_SEARCH_NEIGHBOR) {
                    node = whichnode(node, wall, Vec(x, y, z));
                    if (node < 0) { node = whichnode(0, Vec(x, y, z)); if (fallbacks) (*fallbacks)++; }
                } else {
                    node = whichnode(0, Vec(x, y, z));
                }
                if (node == oldnode) {                       // :418-435 / :476-493
                    x = std::nextafter(x, (kx < 0.0) ? -DBL_MAX : DBL_MAX);
                    y = std::nextafter(y, (ky < 0.0) ? -DBL_MAX : DBL_MAX);
                    z = std::nextafter(z, (kz < 0.0) ? -DBL_MAX : DBL_MAX);
                    node = whichnode(0, Vec(x, y, z));
                    if (node == oldnode) break;
                }
            }
        } else {                                             // Bookkeeping (:500-640), octree only
            int l = node;
            while (true) {
                if (++guard > (1L << 22)) return;   // test guard
                const Box& b = box[l];
                double xnext = (kx < 0.0) ? b.xmin : b.xmax;
                double ynext = (ky < 0.0) ? b.ymin : b.ymax;
                double znext = (kz < 0.0) ? b.zmin : b.zmax;
                double dsx = (std::fabs(kx) > 1e-15) ? (xnext-x)/kx : DBL_MAX;
                double dsy = (std::fabs(ky) > 1e-15) ? (ynext-y)/ky : DBL_MAX;
                double dsz = (std::fabs(kz) > 1e-15) ? (znext-z)/kz : DBL_MAX;
                if (dsx <= dsy && dsx <= dsz) {
                    p.addSegment(cell[l], dsx);
                    x = xnext; y += ky*dsx; z += kz*dsx;
                    while (true) {
                        int oct = ((l-1) % 8) + 1;
                        bool place = (kx < 0.0) ? (oct % 2 == 1) : (oct % 2 == 0);
                        if (!place) break;
                        l = father[l];
                        if (l == 0) return;
                    }
                    l += (kx < 0.0) ? -1 : 1;
                    while (cell[l] == -1) {
                        int c0 = child[l];
                        double yM = box[c0].ymax, zM = box[c0].zmax;
                        if (kx < 0.0) l = (y <= yM) ? ((z <= zM) ? c0+1 : c0+5) : ((z <= zM) ? c0+3 : c0+7);
                        else          l = (y <= yM) ? ((z <= zM) ? c0+0 : c0+4) : ((z <= zM) ? c0+2 : c0+6);
                    }
                } else if (dsy < dsx && dsy <= dsz) {
                    p.addSegment(cell[l], dsy);
                    x += kx*dsy; y = ynext; z += kz*dsy;
                    while (true) {
                        bool place = (ky < 0.0) ? ((l-1) % 4 < 2) : ((l-1) % 4 > 1);
                        if (!place) break;
                        l = father[l];
                        if (l == 0) return;
                    }
                    l += (ky < 0.0) ? -2 : 2;
                    while (cell[l] == -1) {
                        int c0 = child[l];
                        double xM = box[c0].xmax, zM = box[c0].zmax;
                        if (ky < 0.0) l = (x <= xM) ? ((z <= zM) ? c0+2 : c0+6) : ((z <= zM) ? c0+3 : c0+7);
                        else          l = (x <= xM) ? ((z <= zM) ? c0+0 : c0+4) : ((z <= zM) ? c0+1 : c0+5);
                    }
                } else if (dsz < dsx && dsz < dsy) {
                    p.addSegment(cell[l], dsz);
                    x += kx*dsz; y += ky*dsz; z = znext;
                    while (true) {
                        int oct = ((l-1) % 8) + 1;
                        bool place = (kz < 0.0) ? (oct < 5) : (oct > 4);
                        if (!place) break;
                        l = father[l];
                        if (l == 0) return;
                    }
                    l += (kz < 0.0) ? -4 : 4;
                    while (cell[l] == -1) {
                        int c0 = child[l];
                        double xM = box[c0].xmax, yM = box[c0].ymax;
                        if (kz < 0.0) l = (x <= xM) ? ((y <= yM) ? c0+4 : c0+6) : ((y <= yM) ? c0+5 : c0+7);
                        else          l = (x <= xM) ? ((y <= yM) ? c0+0 : c0+2) : ((y <= yM) ? c0+1 : c0+3);
                    }
                } else {
                    return;
                }
            }
        }
    }
};

// VoronoiMesh (SKIRTcore/VoronoiMesh.cpp) over flat arrays.
struct VoronoiGrid : Grid {
    vector<Vec> sites;
    vector<int64_t> noff;
    vector<int> nbr;
    int nb;
    vector<int64_t> boff;
    vector<int> bids;
    vector<double> vol;
    vector<Box> bbox;
    double eps;

    double volume(int m) const override { return vol[m]; }
    int cellIndex(Vec r) const {                                 // VoronoiMesh.cpp:541-570
        if (!ext.contains(r)) return -1;
        int i, j, k;
        ext.cellindices(i, j, k, r, nb, nb, nb);
        int64_t b = (int64_t)i*nb*nb + (int64_t)j*nb + k;
        // nearest site among the cells overlapping this block (the reference's kd-tree search is exact)
        int m = -1; double mdist = DBL_MAX;
        for (int64_t q = boff[b]; q < boff[b+1]; q++) {
            double d = (r - sites[bids[q]]).norm2();
            if (d < mdist) { m = bids[q]; mdist = d; }
        }
        return m;
    }
    int whichcell(Vec r) const override { return cellIndex(r); }
    bool isPointClosestTo(Vec r, int m) const {                  // VoronoiMesh.cpp:640-648
        double target = (r - sites[m]).norm2();
        for (int64_t q = noff[m]; q < noff[m+1]; q++) {
            int id = nbr[q];
            if (id >= 0 && (r - sites[id]).norm2() < target) return false;
        }
        return true;
    }
    Vec randomPositionInCell(int m, Rng& rng) const override {   // VoronoiMesh.cpp:620-636
        for (int i = 0; i < 10000; i++) {
            Vec r = rng.position(bbox[m]);
            if (isPointClosestTo(r, m)) return r;
        }
        return sites[m];
    }
    void path(Path& p, long* fallbacks) const override {        // VoronoiMesh.cpp:778-873
        p.clear();
        Vec k = p.k;
        Vec r;
        if (!p.moveInside(ext, eps, r)) r = Vec(INFINITY, INFINITY, INFINITY);
        int mr = cellIndex(r);
        if (mr < 0) return p.clear();
        long guard = 0;
        while (mr >= 0) {
            if (++guard > (1L << 22)) { if (fallbacks) (*fallbacks)++; break; }   // test guard
            Vec pr = sites[mr];
            double sq = DBL_MAX;
            const int NO_INDEX = -99;
            int mq = NO_INDEX;
            for (int64_t q = noff[mr]; q < noff[mr+1]; q++) {
                int mi = nbr[q];
                double si = 0;
                if (mi >= 0) {
                    Vec pi = sites[mi];
                    Vec n = pi - pr;
                    double ndotk = dot(n, k);
                    if (ndotk > 0) {
                        Vec pp = 0.5 * (pi + pr);
                        si = dot(n, pp - r) / ndotk;
                    }
                } else {
                    switch (mi) {
                        case -1: si = (ext.xmin - r.x)/k.x; break;
                        case -2: si = (ext.xmax - r.x)/k.x; break;
                        case -3: si = (ext.ymin - r.y)/k.y; break;
                        case -4: si = (ext.ymax - r.y)/k.y; break;
                        case -5: si = (ext.zmin - r.z)/k.z; break;
                        case -6: si = (ext.zmax - r.z)/k.z; break;
                        default: si = 0;
                    }
                }
                if (si > 0 && si < sq) { sq = si; mq = mi; }
            }
            if (mq == NO_INDEX) {
                r = r + k*eps;
                mr = cellIndex(r);
                if (fallbacks) (*fallbacks)++;
            } else {
                p.addSegment(mr, sq);
                r = r + (sq+eps)*k;
                mr = mq;
            }
        }
    }
};

// ---------------------------------------------------------------------------------------------
// Special functions

// Lambert W, branch -1, on [-1/e, 0) -- the function SpecialFunctions::LambertW1 evaluates
// (SKIRTcore/SpecialFunctions.cpp:579-630).  Halley iteration on w e^w = z started from the
// branch-point series in p = -sqrt(2(1+e z)) or from the asymptotic form log(-z) - log(-log(-z)),
// iterated to full double precision.
static double lambertW1(double z) {
    if (z == 0.0) return -DBL_MAX;
    const double em1 = 0.36787944117144233;
    double q = z + em1;
    double w;
    if (q < 0.3) {
        double p = -std::sqrt(2.0*M_E*std::max(q, 0.0));
        w = -1.0 + p - p*p/3.0 + 11.0/72.0*p*p*p - 43.0/540.0*p*p*p*p;
    } else {
        double l1 = std::log(-z), l2 = std::log(-l1);
        w = l1 - l2 + l2/l1;
    }
    if (q < 1e-12) return w;
    for (int i = 0; i < 50; i++) {
        double e = std::exp(w);
        double f = w*e - z;
        double wp1 = w + 1.0;
        if (wp1 == 0.0) break;
        double dw = f / (e*wp1 - (w+2.0)*f/(2.0*wp1));
        w -= dw;
        if (std::fabs(dw) <= 1e-15*std::fabs(w)) break;
    }
    return w;
}

// ---------------------------------------------------------------------------------------------
// Geometries

struct Geometry {
    int type;
    double p[6];
    // ExpDisk (ExpDiskGeometry.cpp:24-40)
    double hR, hz, Rmax, zmax, Rmin, rho0;
    // Sersic (SersicGeometry.cpp:29-39, SersicFunction.cpp:17-76)
    double n, reff, srho0;
    vector<double> sv, Sv, Mv;
    // clumpy decorator (ClumpyGeometryDecorator.cpp)
    double f = 0; int N = 0; double h = 0; int cutoff = 0; int kernel = 0;
    vector<Vec> clumps;
    vector<double> kXv;   // cubic spline cumulative table (CubicSplineSmoothingKernel.cpp:22-38)

    void setup(const skg_geometry& g) {
        type = g.type;
        for (int i = 0; i < 6; i++) p[i] = g.p[i];
        if (type == SKG_GEOM_EXPDISK) {
            hR = p[0]; hz = p[1]; Rmax = p[2]; zmax = p[3]; Rmin = p[4];
            double intphi = 2.0*M_PI;
            double intz = (zmax > 0) ? -2.0*hz*std::expm1(-zmax/hz) : 2.0*hz;
            double tmin = (Rmin > 0) ? std::exp(-Rmin/hR)*(1.0+Rmin/hR) : 1.0;
            double tmax = (Rmax > 0) ? std::exp(-Rmax/hR)*(1.0+Rmax/hR) : 0.0;
            double intR = hR*hR*(tmin-tmax);
            rho0 = 1.0/(intR*intphi*intz);
        } else if (type == SKG_GEOM_SERSIC) {
            n = p[0]; reff = p[1];
            srho0 = 1.0/(reff*reff*reff);
            sersicTable();
        }
        if (g.clump_count > 0) {
            f = g.clump_fraction; N = g.clump_count; h = g.clump_radius; cutoff = g.clump_cutoff;
            kernel = g.clump_kernel;
            clumps.resize(N);
            for (int i = 0; i < N; i++) clumps[i] = Vec(g.clump_pos[3*i], g.clump_pos[3*i+1], g.clump_pos[3*i+2]);
            std::stable_sort(clumps.begin(), clumps.end(), [](Vec a, Vec b) { return a.x < b.x; });
            if (kernel == SKG_KERNEL_CUBICSPLINE) {
                int Nu = 400; double du = 1.0/Nu;
                kXv.resize(Nu+1);
                for (int k = 0; k <= Nu; k++) {
                    double u = k*du, u2 = u*u, u3 = u*u2;
                    kXv[k] = (u < 0.5) ? u3*(32.0/3.0 - 192.0/5.0*u2 + 32.0*u3)
                                       : -1.0/15.0 - 64.0*u3*(-1.0/3.0 + 0.75*u - 0.6*u2 + u3/6.0);
                }
            }
        }
    }
    void sersicTable() {                                     // SersicFunction.cpp:17-76
        double b = 2.0*n - 1.0/3.0 + 4.0/405.0/n + 46.0/25515.0/(n*n) + 131.0/1148175.0/(n*n*n);
        double I0 = std::pow(b, 2.0*n) / (M_PI*std::tgamma(2.0*n+1));
        int Ns = 101;
        sv.assign(Ns, 0); Sv.assign(Ns, 0); Mv.assign(Ns, 0);
        double logsmin = -6.0, logsmax = 4.0, dlogs = (logsmax-logsmin)/(Ns-1.0);
        for (int i = 0; i < Ns; i++) {
            double s = std::pow(10.0, logsmin + i*dlogs);
            sv[i] = s;
            double alpha = b*std::pow(s, 1.0/n);
            double sum = 0.0;
            int Nu = 10000; double tmax = 100.0;
            double umax = std::sqrt((tmax+1.0)*(tmax-1.0)), du = umax/Nu;
            for (int j = 0; j <= Nu; j++) {
                double weight = (j == 0 || j == Nu) ? 0.5 : 1.0;
                double u = j*du, u2 = u*u, w;
                if (u > 1e-3) w = (std::pow(1.0+u2, 2.0*n) - 1.0)/u2;
                else w = 2.0*n + n*(2.0*n-1.0)*u2 + 2.0/3.0*n*(2.0*n-1.0)*(n-1.0)*u2*u2;
                sum += weight * 2.0*std::exp(-alpha*(1.0+u2))/std::sqrt(w);
            }
            Sv[i] = I0*std::pow(b, n)*std::pow(alpha, 1.0-n)/M_PI*du*sum;
        }
        for (int i = 1; i < Ns; i++) {
            double sum = 0.0;
            for (int j = 0; j <= 32; j++) {
                double weight = (j == 0 || j == 32) ? 0.5 : 1.0;
                double ds = (sv[i]-sv[i-1])/32.0;
                double s = sv[i-1] + j*ds;
                sum += weight*sersicS(s)*s*s*ds;
            }
            Mv[i] = Mv[i-1] + 4.0*M_PI*sum;
        }
        for (int i = 0; i < Ns; i++) Mv[i] /= Mv[Ns-1];
    }
    double sersicS(double s) const {                         // SersicFunction.cpp:80-92
        int Ns = sv.size();
        if (s <= sv[0]) return Sv[0];
        if (s >= sv[Ns-1]) return Sv[Ns-1];
        int i = locate_clip(sv.data(), Ns, s);
        return interpolate_loglog(s, sv[i], sv[i+1], Sv[i], Sv[i+1]);
    }
    double inversemass(double M) const {                     // SersicFunction.cpp:110-122
        int Ns = sv.size();
        if (M <= Mv[0]) return sv[0];
        if (M >= Mv[Ns-1]) return sv[Ns-1];
        int i = locate_clip(Mv.data(), Ns, M);
        return interpolate_loglog(M, Mv[i], Mv[i+1], sv[i], sv[i+1]);
    }
    double baseDensity(Vec r) const {
        if (type == SKG_GEOM_EXPDISK) {                      // ExpDiskGeometry.cpp:117-129
            double R = std::sqrt(r.x*r.x + r.y*r.y), absz = std::fabs(r.z);
            if (Rmax > 0.0 && R > Rmax) return 0.0;
            if (zmax > 0.0 && absz > zmax) return 0.0;
            if (R < Rmin) return 0.0;
            return rho0*std::exp(-R/hR)*std::exp(-absz/hz);
        } else if (type == SKG_GEOM_SERSIC) {                // SersicGeometry.cpp:72-77
            return srho0*sersicS(r.norm()/reff);
        } else if (type == SKG_GEOM_PLUMMER) {
            double c = p[0], u = r.norm()/c;
            return 3.0/(4.0*M_PI*c*c*c)*std::pow(1.0+u*u, -2.5);
        }
        return r.norm() == 0 ? INFINITY : 0;                 // PointGeometry.cpp:27-32
    }
    double kernelDensity(double u) const {
        if (kernel == SKG_KERNEL_UNIFORM) return (u < 0.0 || u > 1.0) ? 0.0 : 0.75/M_PI;
        if (u < 0.0 || u > 1.0) return 0.0;                  // CubicSplineSmoothingKernel.cpp:42-50
        if (u < 0.5) return 8.0/M_PI*(1.0 - 6.0*u*u*(1.0-u));
        return 8.0/M_PI*2.0*(1.0-u)*(1.0-u)*(1.0-u);
    }
    double kernelRadius(Rng& rng) const {
        double X = rng.uniform();
        if (kernel == SKG_KERNEL_UNIFORM) return std::pow(X, 1.0/3.0);
        int Nu = kXv.size()-1;                               // CubicSplineSmoothingKernel.cpp:54-61
        int k = locate_clip(kXv.data(), Nu+1, X);
        double pp = (X-kXv[k])/(kXv[k+1]-kXv[k]);
        return (k+pp)/Nu;
    }
    // NR::locate on the clump vector ordered by x (NR.hpp:76-95), as used by
    // ClumpyGeometryDecorator::density (ClumpyGeometryDecorator.cpp:142-143)
    int locateClump(double x) const {
        int nn = clumps.size();
        if (x < clumps[0].x) return -1;
        if (clumps[nn-1].x < x) return nn-1;
        int jl = -1, ju = nn;
        while (ju-jl > 1) { int jm = (ju+jl) >> 1; if (x < clumps[jm].x) ju = jm; else jl = jm; }
        if (jl <= 0) return 0;
        if (jl >= nn-2) return nn-2;
        return jl;
    }
    double density(Vec r) const {
        if (N == 0) return baseDensity(r);
        double rhosmooth = (1.0-f)*baseDensity(r);           // ClumpyGeometryDecorator.cpp:136-154
        if (cutoff && !rhosmooth) return 0.0;
        double rhoclumpy = 0.0, Mclump = f/N;
        int istart = std::max(0, locateClump(r.x - h));
        int iend = std::max(0, locateClump(r.x + h));
        for (int i = istart; i <= iend; i++) {
            double u = (r - clumps[i]).norm()/h;
            rhoclumpy += Mclump*kernelDensity(u)/std::pow(h, 3);
        }
        return rhosmooth + rhoclumpy;
    }
    Vec basePosition(Rng& rng) const {
        if (type == SKG_GEOM_EXPDISK) {                      // SepAxGeometry.cpp:20-30
            double R, X;
            do {                                             // ExpDiskGeometry.cpp:133-144
                X = rng.uniform();
                R = hR*(-1.0 - lambertW1((X-1.0)/M_E));
            } while ((Rmax > 0.0 && R >= Rmax) || R <= Rmin);
            double phi = 2.0*M_PI*rng.uniform();
            double z;
            do {                                             // ExpDiskGeometry.cpp:148-161
                X = rng.uniform();
                z = (X <= 0.5) ? hz*std::log(2.0*X) : -hz*std::log(2.0*(1.0-X));
            } while (zmax > 0.0 && std::fabs(z) >= zmax);
            return Vec(R*std::cos(phi), R*std::sin(phi), z);  // Position.cpp:24-31
        } else if (type == SKG_GEOM_SERSIC || type == SKG_GEOM_PLUMMER) {  // SpheGeometry.cpp:36-44
            double rr;
            if (type == SKG_GEOM_SERSIC) rr = reff*inversemass(rng.uniform());  // SersicGeometry.cpp:84-90
            else { double X = rng.uniform(); rr = p[0]/std::sqrt(std::pow(X, -2.0/3.0) - 1.0); }
            Vec k = rng.direction();
            return rr*k;
        }
        return Vec();                                        // PointGeometry.cpp:36-41
    }
    Vec generatePosition(Rng& rng) const {
        if (N == 0) return basePosition(rng);
        while (true) {                                       // ClumpyGeometryDecorator.cpp:158-177
            double X = rng.uniform();
            if (X > f) return basePosition(rng);
            int i = std::min(static_cast<int>((X/f)*N), N-1);
            double u = kernelRadius(rng);
            Vec k = rng.direction();
            Vec r = clumps[i] + u*h*k;
            if (!cutoff || baseDensity(r)) return r;
        }
    }
};

// ---------------------------------------------------------------------------------------------
// Instruments (DistantInstrument.cpp:27-50, SingleFrameInstrument.cpp:26-42,130-147)

struct Instrument {
    int type;
    double costheta, sintheta, cosphi, sinphi, cospa, sinpa;
    Vec kobs;
    int Nxp = 0, Nyp = 0;
    double xpmin, ypmin, xpsiz, ypsiz;
    int nscatt_levels = 0;
    int ncomp = 1;
    vector<double> cube, sed;    // [ncomp][nlambda][Nyp][Nxp], [ncomp][nlambda]
    std::mutex* lock = nullptr;

    void setup(const skg_instrument& in, int nlambda, int nstellar) {
        type = in.type;
        costheta = std::cos(in.inclination); sintheta = std::sin(in.inclination);
        cosphi = std::cos(in.azimuth); sinphi = std::sin(in.azimuth);
        cospa = std::cos(in.position_angle); sinpa = std::sin(in.position_angle);
        kobs = Rng::dirFromAngles(in.inclination, in.azimuth);
        if (type != SKG_INSTR_SED) {
            Nxp = in.nxp; Nyp = in.nyp;
            xpmin = in.xc - 0.5*in.fovx; xpsiz = in.fovx/Nxp;
            ypmin = in.yc - 0.5*in.fovy; ypsiz = in.fovy/Nyp;
        }
        if (type == SKG_INSTR_FULL) { nscatt_levels = in.nscatt_levels; ncomp = SKG_FULL_NBASE + nscatt_levels; }
        if (type == SKG_INSTR_FRAME && in.stellar_comps) ncomp = 1 + nstellar;   // MultiFrameInstrument.cpp:17-57
        if (type != SKG_INSTR_SED) cube.assign((size_t)ncomp*nlambda*Nxp*Nyp, 0.0);
        sed.assign((size_t)ncomp*nlambda, 0.0);
    }
    int pixel(Vec r) const {                                 // SingleFrameInstrument.cpp:130-147
        double x = r.x, y = r.y, z = r.z;
        double xpp = -sinphi*x + cosphi*y;
        double ypp = -cosphi*costheta*x - sinphi*costheta*y + sintheta*z;
        double xp = cospa*xpp - sinpa*ypp;
        double yp = sinpa*xpp + cospa*ypp;
        int i = static_cast<int>(std::floor((xp-xpmin)/xpsiz));
        int j = static_cast<int>(std::floor((yp-ypmin)/ypsiz));
        if (i < 0 || i >= Nxp || j < 0 || j >= Nyp) return -1;
        return i + Nxp*j;
    }
};

static inline void atomic_add(double& target, double value) {   // LockFree.hpp:22-34
    std::atomic_ref<double> a(target);
    double old = a.load(std::memory_order_relaxed);
    while (!a.compare_exchange_weak(old, old+value, std::memory_order_relaxed)) {}
}

// ---------------------------------------------------------------------------------------------
// Simulation state

struct Stats { std::atomic<long> packets{0}, steps{0}, traversals{0}, scatterings{0}, fallbacks{0}; };

struct Sim {
    Grid* grid = nullptr;
    int nlambda = 0;
    vector<double> lambda, dlambda;
    int ncomp = 0;
    vector<vector<double>> kext, kabs, ksca, albedo, g;   // [h][ell]
    vector<double> rho;                                   // [h*ncells + m]
    vector<Geometry> dustgeom; vector<double> dustnorm;
    vector<Geometry> stargeom; vector<vector<double>> starL;
    vector<double> Lv; vector<vector<double>> Xvv;        // StellarSystem.cpp:35-52
    double emissionBias = 0.5;
    vector<Instrument> instr;
    double minWeightReduction = 1e4; int minfs = 0; double xi = 0.5;
    bool storeAbs = false;
    vector<double> LabsStel, LabsDust;                    // [m*nlambda + ell]
    // dust emission
    bool dustEmission = false; double dustEmissionBias = 0.5;
    vector<double> Tv; vector<double> planckabs;           // single component grey body
    vector<double> Lvv;                                   // normalised emission spectra [m*nlambda+ell]
    vector<double> Labsbol, Tcell;
    Stats stats;

    double density(int m, int h) const { return m >= 0 ? rho[(size_t)h*grid->ncells + m] : 0; }
    double kapparho(int m, int ell) const {               // DustSystem.cpp:459-485
        double r = 0;
        for (int h = 0; h < ncomp; h++) r += kext[h][ell]*density(m, h);
        return r;
    }
    double opticaldepth(Path& p, int ell) {               // DustSystem.cpp:960-976
        grid->path(p, nullptr);
        stats.steps += p.v.size(); stats.traversals++;
        return p.opticalDepth([&](int m) { return kapparho(m, ell); });
    }
    void fillOpticalDepth(Path& p, int ell) {             // DustSystem.cpp:935-956
        grid->path(p, nullptr);
        stats.steps += p.v.size(); stats.traversals++;
        p.fillOpticalDepth([&](int m) { return kapparho(m, ell); });
    }
};

struct Packet {          // PhotonPackage (PhotonPackage.hpp:28-139)
    double L; int ell; Vec r, k; int nscatt; int stellar;
};

// Instrument::detect for the four instrument types (SEDInstrument.cpp:32-42, FrameInstrument.cpp:33-47,
// SimpleInstrument.cpp:35-49, FullInstrument.cpp:109-177).
static void detect(Sim& S, Instrument& I, const Packet& pp, Path& path) {
    const int nl = S.nlambda;
    path.r = pp.r; path.k = pp.k;
    if (I.type == SKG_INSTR_FRAME) {
        int l = I.pixel(pp.r);
        if (l >= 0) {
            double taupath = S.opticaldepth(path, pp.ell);
            const size_t fp = (size_t)I.Nxp*I.Nyp;
            atomic_add(I.cube[(size_t)pp.ell*fp + l], pp.L*std::exp(-taupath));
            // the frame of the packet's stellar component (writeStellarComps)
            if (I.ncomp > 1 && pp.stellar >= 0)
                atomic_add(I.cube[((size_t)(1 + pp.stellar)*nl + pp.ell)*fp + l], pp.L*std::exp(-taupath));
        }
        return;
    }
    int l = (I.type == SKG_INSTR_SED) ? -1 : I.pixel(pp.r);
    double taupath = S.opticaldepth(path, pp.ell);
    double Lextf = pp.L*std::exp(-taupath);
    size_t fp = (size_t)I.Nxp*I.Nyp;
    if (I.type == SKG_INSTR_SED || I.type == SKG_INSTR_SIMPLE) {
        atomic_add(I.sed[pp.ell], Lextf);
        if (l >= 0) atomic_add(I.cube[(size_t)pp.ell*fp + l], Lextf);
        return;
    }
    // FullInstrument: component c at sed[c*nl+ell], cube[(c*nl+ell)*fp + l]; component 0 = total
    auto add = [&](int c, double v) {
        atomic_add(I.sed[(size_t)c*nl + pp.ell], v);
        if (l >= 0) atomic_add(I.cube[((size_t)c*nl + pp.ell)*fp + l], v);
    };
    add(SKG_FULL_TOT, Lextf);
    if (pp.stellar >= 0) {
        if (pp.nscatt == 0) { add(SKG_FULL_TRA, pp.L); if (S.ncomp) add(SKG_FULL_STRDIR, Lextf); }
        else {
            add(SKG_FULL_STRSCA, Lextf);
            if (pp.nscatt <= I.nscatt_levels) add(SKG_FULL_NBASE + pp.nscatt - 1, Lextf);
        }
    } else {
        if (pp.nscatt == 0) add(SKG_FULL_DUSDIR, Lextf); else add(SKG_FULL_DUSSCA, Lextf);
    }
}

static void peeloffemission(Sim& S, const Packet& pp, Path& path) {   // MonteCarloSimulation.cpp:299-309
    for (auto& I : S.instr) {
        Packet ppp = pp; ppp.k = I.kobs; ppp.nscatt = 0;
        detect(S, I, ppp, path);
    }
}

static double phaseFunctionValue(const Sim& S, int h, const Packet& pp, Vec kobs) {  // DustMix.cpp:648-654
    double cosalpha = dot(pp.k, kobs);
    double g = S.g[h][pp.ell];
    double t = 1.0 + g*g - 2*g*cosalpha;
    return (1.0-g)*(1.0+g)/std::sqrt(t*t*t);
}

static void peeloffscattering(Sim& S, const Packet& pp, Path& path) {  // MonteCarloSimulation.cpp:313-357
    int Ncomp = S.ncomp;
    double wv[8];
    if (Ncomp == 1) wv[0] = 1.0;
    else {
        int m = S.grid->whichcell(pp.r);
        if (m == -1) return;
        double sum = 0;
        for (int h = 0; h < Ncomp; h++) { wv[h] = S.ksca[h][pp.ell]*S.density(m, h); sum += wv[h]; }
        if (sum <= 0) return;
        for (int h = 0; h < Ncomp; h++) wv[h] /= sum;
    }
    for (auto& I : S.instr) {
        double Iw = 0;
        for (int h = 0; h < Ncomp; h++) Iw += wv[h]*phaseFunctionValue(S, h, pp, I.kobs);
        Packet ppp = pp; ppp.k = I.kobs; ppp.L = pp.L*Iw; ppp.nscatt = pp.nscatt + 1;
        detect(S, I, ppp, path);
    }
}

static void simulateescapeandabsorption(Sim& S, Packet& pp, Path& path, bool store) {  // :432-509
    double taupath = path.tau();
    int ell = pp.ell;
    double L = pp.L;
    bool stellar = pp.stellar >= 0;
    vector<double>& Labs = stellar ? S.LabsStel : S.LabsDust;
    if (S.ncomp == 1) {
        double albedo = S.albedo[0][ell];
        double expfactor = -std::expm1(-taupath);
        if (store) {
            int N = path.v.size();
            for (int n = 0; n < N; n++) {
                int m = path.v[n].m;
                if (m != -1) {
                    double taustart = (n == 0) ? 0.0 : path.v[n-1].tau;
                    double expfactorm = -std::expm1(-path.v[n].dtau);
                    double Lintm = L*std::exp(-taustart)*expfactorm;
                    atomic_add(Labs[(size_t)m*S.nlambda + ell], (1.0-albedo)*Lintm);
                }
            }
        }
        pp.L = L*albedo*expfactor;
    } else {
        double Lsca = 0.0;
        int N = path.v.size();
        for (int n = 0; n < N; n++) {
            int m = path.v[n].m;
            if (m != -1) {
                double ksca = 0.0, kext = 0.0;
                for (int h = 0; h < S.ncomp; h++) {
                    double r = S.density(m, h);
                    ksca += r*S.ksca[h][ell]; kext += r*S.kext[h][ell];
                }
                double albedo = (kext > 0.0) ? ksca/kext : 0.0;
                double taustart = (n == 0) ? 0.0 : path.v[n-1].tau;
                double expfactorm = -std::expm1(-path.v[n].dtau);
                double Lintm = L*std::exp(-taustart)*expfactorm;
                Lsca += albedo*Lintm;
                if (store) atomic_add(Labs[(size_t)m*S.nlambda + ell], (1.0-albedo)*Lintm);
            }
        }
        pp.L = Lsca;
    }
}

static void simulatepropagation(Sim& S, Packet& pp, Path& path, Rng& rng) {   // :513-531
    double taupath = path.tau();
    if (taupath == 0.0) return;
    double tau;
    if (S.xi == 0.0) tau = rng.exponcutoff(taupath);
    else {
        double X = rng.uniform();
        tau = (X < S.xi) ? rng.uniform()*taupath : rng.exponcutoff(taupath);
        double p = -std::exp(-tau)/std::expm1(-taupath);
        double q = (1.0-S.xi)*p + S.xi/taupath;
        pp.L *= p/q;
    }
    double s = path.pathlength(tau);
    pp.r = pp.r + s*pp.k;
}

static void simulatescattering(Sim& S, Packet& pp, Rng& rng) {   // :535-543, DustSystem.cpp:855-869
    int h = 0;
    if (S.ncomp > 1) {
        int m = S.grid->whichcell(pp.r);
        if (m >= 0) {
            vector<double> pv(S.ncomp), Xv;
            for (int c = 0; c < S.ncomp; c++) pv[c] = S.ksca[c][pp.ell]*S.density(m, c);
            cdf(Xv, pv);
            h = locate_clip(Xv.data(), Xv.size(), rng.uniform());
        }
    }
    double g = S.g[h][pp.ell];                                   // DustMix.cpp:595-602
    Vec knew;
    if (std::fabs(g) < 1e-6) knew = rng.direction();
    else {
        double f = ((1.0-g)*(1.0+g))/(1.0-g+2.0*g*rng.uniform());
        double costheta = (1.0+g*g-f*f)/(2.0*g);
        knew = rng.direction(pp.k, costheta);
    }
    pp.nscatt++; pp.k = knew;                                   // PhotonPackage.cpp:98-103
}

// The loop body shared by the stellar and dust emission chunks (MonteCarloSimulation.cpp:277-288,
// PanMonteCarloSimulation.cpp:325-338).
static void lifecycle(Sim& S, Packet& pp, Path& path, Path& ppath, Rng& rng, double Lthreshold,
                      bool store, bool peel) {
    if (peel) peeloffemission(S, pp, ppath);
    if (S.ncomp == 0) return;
    while (true) {
        path.r = pp.r; path.k = pp.k;
        S.fillOpticalDepth(path, pp.ell);
        double tau = path.tau();
        if (tau < 0.0 || std::isnan(tau) || std::isinf(tau)) { pp.L = 0; return; }
        simulateescapeandabsorption(S, pp, path, store);
        if (pp.L <= 0 || (pp.L <= Lthreshold && pp.nscatt >= S.minfs)) break;
        simulatepropagation(S, pp, path, rng);
        if (peel) peeloffscattering(S, pp, ppath);
        simulatescattering(S, pp, rng);
        S.stats.scatterings++;
    }
}

static void stellarLaunch(Sim& S, Packet& pp, int ell, double L, Rng& rng) {   // StellarSystem.cpp:116-158
    int N = S.stargeom.size();
    int h = 0;
    double Lh_launch;
    if (N == 1) { Lh_launch = L; }
    else {
        double X = rng.uniform();
        if (X < S.emissionBias) h = std::max(0, std::min(N-1, static_cast<int>(N*X/S.emissionBias)));
        else h = locate_clip(S.Xvv[ell].data(), N+1, (X-S.emissionBias)/(1.0-S.emissionBias));
        double Lh = S.starL[h][ell];
        if (!(Lh > 0)) { pp = Packet{0., ell, Vec(), Vec(), 0, h}; return; }
        double Lmean = S.Lv[ell]/N;
        Lh_launch = L*(1.0/(1.0 - S.emissionBias + S.emissionBias*Lmean/Lh));
    }
    Vec r = S.stargeom[h].generatePosition(rng);                 // GeometricStellarComp.cpp:75-81
    Vec k = rng.direction();
    pp = Packet{Lh_launch, ell, r, k, 0, h};
}

// MonteCarloSimulation::setChunkParams (MonteCarloSimulation.cpp:68-114), task-parallel mode.
static void chunkParams(double packages, int Nthreads, int Nprocs, int Nlambda,
                        uint64_t& Nchunks, uint64_t& chunksize, uint64_t& Npp) {
    if (packages <= 0) { Nchunks = chunksize = Npp = 0; return; }
    long totalChunks;
    if (Nthreads == 1) totalChunks = 1;
    else totalChunks = (long)std::ceil(std::max(10.*double(Nthreads*Nprocs)/Nlambda, packages/1e7));
    if (totalChunks % Nprocs) totalChunks = totalChunks + Nprocs - (totalChunks % Nprocs);
    chunksize = (uint64_t)std::ceil(packages/totalChunks);
    Nchunks = totalChunks/Nprocs;
    Npp = totalChunks*chunksize;
}

// Parallel::call over (Nlambda x Nchunks) indices with dynamic grabbing (Parallel.cpp:169-199);
// thread t owns Rng seeded seed+t (Random.cpp:41-56).
template<typename F> static void parallelCall(int nthreads, uint64_t nitems, uint64_t seed, F body) {
    std::atomic<uint64_t> next{0};
    auto worker = [&](int t) {
        Rng rng; rng.init(seed + t);
        while (true) {
            uint64_t i = next.fetch_add(1);
            if (i >= nitems) break;
            body(i, rng);
        }
    };
    vector<std::thread> th;
    for (int t = 1; t < nthreads; t++) th.emplace_back(worker, t);
    worker(0);
    for (auto& t : th) t.join();
}

// PanMonteCarloSimulation dust emission spectra: DustSystem::meanintensityv (DustSystem.cpp:911-931),
// DustMix::equilibrium (DustMix.cpp:689-697, invplanckabs :674-680), grey body
// (GreyBodyDustEmissivity.cpp:21-45), normalised luminosities (DustLib.cpp:135-148).  One component.
static double planck(double lambda, double T) {   // PlanckFunction.cpp:24-33
    const double h = 6.62606957e-34, c = 2.99792458e8, k = 1.3806488e-23;
    double x = h*c/(lambda*k*T);
    return 2.0*h*c*c/std::pow(lambda, 5)/(std::exp(x) - 1.0);
}
static void calcDustEmission(Sim& S) {
    int Nc = S.grid->ncells, nl = S.nlambda, nT = S.Tv.size();
    S.Lvv.assign((size_t)Nc*nl, 0.0);
    S.Labsbol.assign(Nc, 0.0);
    S.Tcell.assign(Nc, 0.0);
    for (int m = 0; m < Nc; m++) {
        double lb = 0;
        for (int ell = 0; ell < nl; ell++) lb += S.LabsStel[(size_t)m*nl+ell] + S.LabsDust[(size_t)m*nl+ell];
        S.Labsbol[m] = lb;
        // mean intensity and the Planck-abs integral sum_ell sigma_abs J dlambda
        double fac = 4.0*M_PI*S.grid->volume(m);
        double pa = 0.0;
        for (int ell = 0; ell < nl; ell++) {
            double kar = S.kabs[0][ell]*S.density(m, 0);
            double J = (S.LabsStel[(size_t)m*nl+ell] + S.LabsDust[(size_t)m*nl+ell])/(kar*fac)/S.dlambda[ell];
            if (!std::isfinite(J)) J = 0.0;
            pa += S.kabs[0][ell]*J*S.dlambda[ell];
        }
        int p = locate_clip(S.planckabs.data(), nT, pa);
        double T = interpolate_linlin(pa, S.planckabs[p], S.planckabs[p+1], S.Tv[p], S.Tv[p+1]);
        S.Tcell[m] = T;
        double total = 0;
        double* Lv = &S.Lvv[(size_t)m*nl];
        for (int ell = 0; ell < nl; ell++) {
            Lv[ell] = (T > 0) ? S.kabs[0][ell]*planck(S.lambda[ell], T)*S.dlambda[ell] : 0.0;
            total += Lv[ell];
        }
        if (total > 0) for (int ell = 0; ell < nl; ell++) Lv[ell] /= total;
    }
}

static Sim* buildSim(const skg_scene* sc) {
    Sim* S = new Sim();
    const skg_grid& g = sc->grid;
    Box ext{g.xmin, g.ymin, g.zmin, g.xmax, g.ymax, g.zmax};
    double diag = std::sqrt((ext.xmax-ext.xmin)*(ext.xmax-ext.xmin) + (ext.ymax-ext.ymin)*(ext.ymax-ext.ymin)
                            + (ext.zmax-ext.zmin)*(ext.zmax-ext.zmin));
    if (g.type == SKG_GRID_CARTESIAN) {
        auto* G = new CartesianGrid();
        G->Nx = g.nx; G->Ny = g.ny; G->Nz = g.nz;
        G->xv.assign(g.xv, g.xv+g.nx+1); G->yv.assign(g.yv, g.yv+g.ny+1); G->zv.assign(g.zv, g.zv+g.nz+1);
        G->ncells = g.nx*g.ny*g.nz;
        S->grid = G;
    } else if (g.type == SKG_GRID_OCTREE || g.type == SKG_GRID_BINTREE) {
        auto* G = new TreeGrid();
        int n = g.nnodes;
        G->nnodes = n;
        G->box.resize(n);
        for (int l = 0; l < n; l++) {
            const double* b = g.node_box + 6*l;
            G->box[l] = Box{b[0], b[1], b[2], b[3], b[4], b[5]};
        }
        G->child.assign(g.node_child, g.node_child+n);
        G->father.assign(g.node_father, g.node_father+n);
        G->cell.assign(g.node_cell, g.node_cell+n);
        G->dir.assign(g.node_dir, g.node_dir+n);
        if (g.nbr_offsets) {
            G->nbroff.assign(g.nbr_offsets, g.nbr_offsets + 6*(size_t)n + 1);
            G->nbr.assign(g.nbr_ids, g.nbr_ids + G->nbroff.back());
        }
        int nc = 0;
        for (int l = 0; l < n; l++) if (G->cell[l] >= 0) nc++;
        G->idv.assign(nc, 0);
        for (int l = 0; l < n; l++) if (G->cell[l] >= 0) G->idv[G->cell[l]] = l;
        G->ncells = nc;
        G->search = g.search_method;
        G->eps = 1e-12*diag;                                   // TreeDustGrid.cpp:74
        S->grid = G;
    } else {
        auto* G = new VoronoiGrid();
        int n = g.nsites;
        G->sites.resize(n);
        for (int m = 0; m < n; m++) G->sites[m] = Vec(g.sites[3*m], g.sites[3*m+1], g.sites[3*m+2]);
        G->noff.assign(g.vnbr_offsets, g.vnbr_offsets+n+1);
        G->nbr.assign(g.vnbr_ids, g.vnbr_ids + G->noff.back());
        G->nb = g.nb;
        size_t nb3 = (size_t)g.nb*g.nb*g.nb;
        G->boff.assign(g.block_offsets, g.block_offsets+nb3+1);
        G->bids.assign(g.block_ids, g.block_ids + G->boff.back());
        if (g.cell_volume) G->vol.assign(g.cell_volume, g.cell_volume+n); else G->vol.assign(n, 0.0);
        G->bbox.resize(n);
        for (int m = 0; m < n; m++) {
            if (g.cell_bbox) { const double* b = g.cell_bbox + 6*m; G->bbox[m] = Box{b[0], b[1], b[2], b[3], b[4], b[5]}; }
            else G->bbox[m] = ext;
        }
        G->ncells = n;
        G->eps = 1e-12*diag;                                   // VoronoiMesh.cpp:220
        S->grid = G;
    }
    S->grid->ext = ext;

    S->nlambda = sc->nlambda;
    S->lambda.assign(sc->lambda, sc->lambda + sc->nlambda);
    S->dlambda.assign(sc->dlambda, sc->dlambda + sc->nlambda);
    S->ncomp = sc->ncomp;
    for (int h = 0; h < sc->ncomp; h++) {
        const skg_dust_comp& d = sc->dust[h];
        vector<double> ke(d.kappaext, d.kappaext+sc->nlambda), al(d.albedo, d.albedo+sc->nlambda),
                       gg(d.asymmpar, d.asymmpar+sc->nlambda), ka(sc->nlambda), ks(sc->nlambda);
        for (int l = 0; l < sc->nlambda; l++) { ka[l] = ke[l]*(1.-al[l]); ks[l] = ke[l]*al[l]; }  // SimpleOligoDustMix.cpp:38-45
        S->kext.push_back(ke); S->albedo.push_back(al); S->g.push_back(gg); S->kabs.push_back(ka); S->ksca.push_back(ks);
        Geometry G; G.setup(d.geometry); S->dustgeom.push_back(G); S->dustnorm.push_back(d.norm);
    }
    S->emissionBias = sc->emission_bias;
    for (int c = 0; c < sc->nstellar; c++) {
        Geometry G; G.setup(sc->stellar[c].geometry); S->stargeom.push_back(G);
        S->starL.emplace_back(sc->stellar[c].luminosity, sc->stellar[c].luminosity + sc->nlambda);
    }
    int Nst = sc->nstellar;
    S->Lv.assign(sc->nlambda, 0.0);
    S->Xvv.resize(sc->nlambda);
    for (int ell = 0; ell < sc->nlambda; ell++) {
        vector<double> pv(Nst);
        for (int h = 0; h < Nst; h++) { S->Lv[ell] += S->starL[h][ell]; pv[h] = S->starL[h][ell]; }
        if (Nst) cdf(S->Xvv[ell], pv);
    }
    S->instr.resize(sc->ninstr);
    for (int i = 0; i < sc->ninstr; i++) S->instr[i].setup(sc->instr[i], sc->nlambda, sc->nstellar);
    S->minWeightReduction = sc->min_weight_reduction > 0 ? sc->min_weight_reduction : 1e4;
    S->minfs = sc->min_scatt_events;
    S->xi = sc->scatt_bias;
    S->storeAbs = sc->store_absorption || sc->dust_emission;
    if (sc->dust_emission && S->ncomp) {
        // DustMix temperature grid and Planck-integrated absorption (DustMix.cpp:239-263):
        // NR::powgrid(Tv, 0, 5000, 1000, 500) (NR.hpp:189-204)
        const int NT = 1000;
        S->Tv.assign(NT+1, 0.0);
        double q = std::pow(500.0, 1./(NT-1)), qn = std::pow(q, NT);
        for (int i = 0; i <= NT; ++i) S->Tv[i] = 0.0 + (1.-std::pow(q, i))/(1.-qn)*5000.0;
        S->planckabs.assign(NT+1, 0.0);
        for (int p = 1; p <= NT; p++) {
            double pa = 0.0;
            for (int ell = 0; ell < S->nlambda; ell++)
                pa += S->kabs[0][ell]*planck(S->lambda[ell], S->Tv[p])*S->dlambda[ell];
            S->planckabs[p] = pa;
        }
    }
    S->dustEmission = sc->dust_emission;
    S->dustEmissionBias = sc->dust_emission_bias;
    size_t nc = S->grid->ncells;
    S->LabsStel.assign(nc*sc->nlambda, 0.0);
    S->LabsDust.assign(nc*sc->nlambda, 0.0);
    return S;
}

// DustSystem::setSampleDensityBody (DustSystem.cpp:145-172): average of Nrandom samples per cell.
static void sampleDensity(Sim& S, int Nrandom, int nthreads, uint64_t seed) {
    size_t nc = S.grid->ncells;
    S.rho.assign(nc*S.ncomp, 0.0);
    uint64_t nchunks = (nc + 4095)/4096;
    parallelCall(nthreads, nchunks, seed, [&](uint64_t c, Rng& rng) {
        for (size_t m = c*4096; m < std::min(nc, (size_t)(c+1)*4096); m++) {
            double sumv[8] = {0};
            for (int n = 0; n < Nrandom; n++) {
                Vec r = S.grid->randomPositionInCell((int)m, rng);
                for (int h = 0; h < S.ncomp; h++) sumv[h] += S.dustnorm[h]*S.dustgeom[h].density(r);
            }
            for (int h = 0; h < S.ncomp; h++) S.rho[(size_t)h*nc + m] = sumv[h]/Nrandom;
        }
    });
}


// ---------------------------------------------------------------------------------------------
// Tree construction: TreeDustGrid::setupSelfBefore / subdivide (TreeDustGrid.cpp:80-100,
// 166-230) with the mass-fraction criterion, the node masses of TreeNodeSampleDensityCalculator
// (TreeNodeSampleDensityCalculator.cpp:26-45: Nrandom positions uniform in the node box,
// mass = mean density x volume), the total mass of DustComp::mass (DustComp.cpp:110-114: the
// sum of the components' normalisations), and the children of OctTreeNode::createchildren
// (OctTreeNode.cpp:38-56: eight boxes split at the centre) and BinTreeNode::createchildren
// (BinTreeNode.cpp:40-77: two boxes split at the middle along direction level % 3).  Nodes are
// visited in creation order; children are appended, so the ids follow the reference's.

struct TreeBuild {
    vector<Box> box; vector<int> child, father, level; vector<int8_t> dir; vector<uint8_t> split;
    void split_node(int l, int type) {
        const Box b = box[l];
        int id0 = (int)box.size();
        child[l] = id0; split[l] = 1;
        auto push = [&](const Box& c) {
            box.push_back(c); child.push_back(-1); father.push_back(l); level.push_back(level[l] + 1);
            dir.push_back(-1); split.push_back(0);
        };
        if (type == SKG_GRID_OCTREE) {                            // OctTreeNode.cpp:38-56
            double xc = 0.5*(b.xmin+b.xmax), yc = 0.5*(b.ymin+b.ymax), zc = 0.5*(b.zmin+b.zmax);
            push(Box{b.xmin, b.ymin, b.zmin, xc, yc, zc});
            push(Box{xc, b.ymin, b.zmin, b.xmax, yc, zc});
            push(Box{b.xmin, yc, b.zmin, xc, b.ymax, zc});
            push(Box{xc, yc, b.zmin, b.xmax, b.ymax, zc});
            push(Box{b.xmin, b.ymin, zc, xc, yc, b.zmax});
            push(Box{xc, b.ymin, zc, b.xmax, yc, b.zmax});
            push(Box{b.xmin, yc, zc, xc, b.ymax, b.zmax});
            push(Box{xc, yc, zc, b.xmax, b.ymax, b.zmax});
        } else {                                                   // BinTreeNode.cpp:40-77
            int d = level[l] % 3;
            dir[l] = (int8_t)d;
            Box c0 = b, c1 = b;
            if (d == 0) { double c = 0.5*(b.xmin+b.xmax); c0.xmax = c; c1.xmin = c; }
            else if (d == 1) { double c = 0.5*(b.ymin+b.ymax); c0.ymax = c; c1.ymin = c; }
            else { double c = 0.5*(b.zmin+b.zmax); c0.zmax = c; c1.zmin = c; }
            push(c0); push(c1);
        }
    }
};

static double dust_density(const Sim& S, Vec r) {            // CompDustDistribution / DustComp::density
    double rho = 0;
    for (int h = 0; h < S.ncomp; h++) rho += S.dustnorm[h]*S.dustgeom[h].density(r);
    return rho;
}

}  // namespace orc

// =============================================================================================
// extern "C" surface (ctypes)

using namespace orc;

extern "C" {

typedef struct orc_stats {
    int64_t packets, steps, traversals, scatterings, fallbacks;
    uint64_t npp, chunks;
    double seconds;
} orc_stats;

const char* orc_last_error(void) { return g_err.c_str(); }

int orc_chunk_params(double packages, int nthreads, int nprocs, int nlambda,
                     uint64_t* nchunks, uint64_t* chunksize, uint64_t* npp) {
    chunkParams(packages, nthreads, nprocs, nlambda, *nchunks, *chunksize, *npp);
    return 0;
}

// DustGrid::path for n rays; segments of ray i at offsets[i]..offsets[i+1]-1.  The rays are
// independent: nthreads threads trace contiguous ranges of them into per-range buffers, which are
// then concatenated in ray order (the output does not depend on the thread count).
int orc_trace_paths(const skg_scene* sc, const double* r, const double* k, int64_t n,
                    int32_t* cells, double* ds, int64_t* offsets, int64_t capacity, int64_t* fallbacks,
                    int nthreads) {
    Sim* S = buildSim(sc);
    if (nthreads < 1) nthreads = 1;
    const int64_t nr = std::max<int64_t>(1, std::min<int64_t>(nthreads * 4, n));
    struct Range { vector<int32_t> m; vector<double> d; vector<int64_t> cnt; long fb = 0; };
    vector<Range> R(nr);
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        Path p;
        int64_t q;
        while ((q = next.fetch_add(1)) < nr) {
            Range& g = R[q];
            const int64_t i0 = n*q/nr, i1 = n*(q+1)/nr;
            for (int64_t i = i0; i < i1; i++) {
                p.r = Vec(r[3*i], r[3*i+1], r[3*i+2]); p.k = Vec(k[3*i], k[3*i+1], k[3*i+2]);
                S->grid->path(p, &g.fb);
                g.cnt.push_back((int64_t)p.v.size());
                for (auto& s : p.v) { g.m.push_back(s.m); g.d.push_back(s.ds); }
            }
        }
    };
    vector<std::thread> th;
    for (int t = 1; t < nthreads; t++) th.emplace_back(worker);
    worker();
    for (auto& t : th) t.join();
    int64_t pos = 0, i = 0; long fb = 0;
    for (auto& g : R) {
        size_t j = 0;
        for (int64_t c : g.cnt) {
            offsets[i++] = pos;
            for (int64_t e = 0; e < c; e++, j++, pos++)
                if (pos < capacity) { cells[pos] = g.m[j]; ds[pos] = g.d[j]; }
        }
        fb += g.fb;
    }
    offsets[n] = pos;
    if (fallbacks) *fallbacks = fb;
    delete S->grid; delete S;
    return pos > capacity ? SKG_ERR_CAPACITY : 0;
}

// Instrument::opticalDepth for n rays at wavelength ell with the given densities.
int orc_optical_depth(const skg_scene* sc, const double* r, const double* k, int64_t n, int ell, double* tau) {
    Sim* S = buildSim(sc);
    if (!sc->rho) { g_err = "orc_optical_depth needs scene->rho"; delete S->grid; delete S; return SKG_ERR_INVALID; }
    S->rho.assign(sc->rho, sc->rho + (size_t)S->ncomp*S->grid->ncells);
    Path p;
    for (int64_t i = 0; i < n; i++) {
        p.r = Vec(r[3*i], r[3*i+1], r[3*i+2]); p.k = Vec(k[3*i], k[3*i+1], k[3*i+2]);
        tau[i] = S->opticaldepth(p, ell);
    }
    delete S->grid; delete S;
    return 0;
}

// DustGridPath::pathlength restated, for segments of lengths ds[] in cells 0..n-1 with
// kappa*rho kr[] per cell (pinned against the reference TU).
double orc_pathlength(const double* ds, const double* kr, int n, double tau) {
    Path p;
    for (int i = 0; i < n; i++) p.addSegment(i, ds[i]);
    p.fillOpticalDepth([kr](int m) { return kr[m]; });
    return p.pathlength(tau);
}

// DustGridPath::moveInside restated; returns the number of entry segments or -1 for OUTSIDE.
int orc_moveinside(const double* box, double eps, const double* r, const double* k, double* out_r, double* seg) {
    Path p;
    p.r = Vec(r[0], r[1], r[2]); p.k = Vec(k[0], k[1], k[2]);
    Box b{box[0], box[1], box[2], box[3], box[4], box[5]};
    Vec q;
    bool ok = p.moveInside(b, eps, q);
    for (size_t i = 0; i < p.v.size(); i++) seg[i] = p.v[i].ds;
    if (!ok) { out_r[0] = out_r[1] = out_r[2] = INFINITY; return -1; }
    out_r[0] = q.x; out_r[1] = q.y; out_r[2] = q.z;
    return (int)p.v.size();
}

// Sersic profile, cumulative mass and inverse mass at the given points (restated tables).
void orc_sersic(double n, const double* s, int ns, double* S, double* M, const double* X, int nx, double* inv) {
    skg_geometry g; std::memset(&g, 0, sizeof(g));
    g.type = SKG_GEOM_SERSIC; g.p[0] = n; g.p[1] = 1.0;
    Geometry G; G.setup(g);
    int Ns = G.sv.size();
    for (int i = 0; i < ns; i++) {
        S[i] = G.sersicS(s[i]);
        double x = s[i];
        if (x <= G.sv[0]) M[i] = G.Mv[0];
        else if (x >= G.sv[Ns-1]) M[i] = G.Mv[Ns-1];
        else { int j = locate_clip(G.sv.data(), Ns, x); M[i] = interpolate_loglog(x, G.sv[j], G.sv[j+1], G.Mv[j], G.Mv[j+1]); }
    }
    for (int i = 0; i < nx; i++) inv[i] = G.inversemass(X[i]);
}

double orc_lambertw1(double z) { return lambertW1(z); }

// Samples positions from a geometry (launch sampler) with the reference RNG.
int orc_sample_positions(const skg_geometry* g, int64_t n, uint64_t seed, double* out) {
    Geometry G; G.setup(*g);
    Rng rng; rng.init(seed);
    for (int64_t i = 0; i < n; i++) {
        Vec r = G.generatePosition(rng);
        out[3*i] = r.x; out[3*i+1] = r.y; out[3*i+2] = r.z;
    }
    return 0;
}

int orc_density(const skg_geometry* g, const double* r, int64_t n, double* out) {
    Geometry G; G.setup(*g);
    for (int64_t i = 0; i < n; i++) out[i] = G.density(Vec(r[3*i], r[3*i+1], r[3*i+2]));
    return 0;
}

int orc_sample_density(const skg_scene* sc, int nthreads, uint64_t seed, double* rho) {
    Sim* S = buildSim(sc);
    sampleDensity(*S, sc->density_samples > 0 ? sc->density_samples : 100, nthreads, seed);
    std::memcpy(rho, S->rho.data(), S->rho.size()*sizeof(double));
    delete S->grid; delete S;
    return 0;
}


// TreeDustGrid construction (see TreeBuild above).  sampler 0: the reference's Random::position
// (Random.cpp:227-235) from one MT19937 stream seeded `seed`, node after node and sample after
// sample (the order of a single-threaded run); sampler 1: one counter-based stream per node and
// sample, the sampler of the library's device builder (identical node masses, so identical
// decisions).  Writes, in node creation order, the split flags, boxes, first-child ids, fathers,
// cell numbers (leaves in node order, TreeDustGrid.cpp:107-119; -1 otherwise), split directions
// (k-d tree) and levels.  *nnodes receives the node count; SKG_ERR_CAPACITY when it exceeds
// max_nodes (nothing else is written then).
int orc_tree_build(const skg_scene* sc, int type, int minlevel, int maxlevel, double maxfrac, int Nrandom,
                   uint64_t seed, int sampler, int nthreads, int64_t max_nodes, uint8_t* split, double* box,
                   int32_t* child, int32_t* father, int32_t* cell, int8_t* dir, int32_t* level, int64_t* nnodes) {
    Sim* S = buildSim(sc);
    double total = 0;
    for (int h = 0; h < S->ncomp; h++) total += S->dustnorm[h];
    TreeBuild T;
    T.box.push_back(S->grid->ext); T.child.push_back(-1); T.father.push_back(-1); T.level.push_back(0);
    T.dir.push_back(-1); T.split.push_back(0);
    Rng rng; rng.init(seed);
    const bool nocrit = !(maxfrac > 0);
    vector<double> mass;
    size_t l = 0;
    while (l < T.box.size()) {
        // the nodes of one level are contiguous in creation order; their masses are independent of
        // one another (sampler 1), so a level is sampled by several threads at once
        size_t lend = l;
        while (lend < T.box.size() && T.level[lend] == T.level[l]) lend++;
        const int lev = T.level[l];
        if (lev > minlevel && lev < maxlevel && !nocrit) {
            mass.assign(lend - l, 0.0);
            auto body = [&](size_t q) {
                const Box& b = T.box[q];
                double sum = 0;
                if (sampler == 1) {
                    for (int n = 0; n < Nrandom; n++) {
                        Philox ph(seed, (uint64_t)q, 0x7EE0000u + (uint32_t)n);
                        double x = ph.uniform(), y = ph.uniform(), z = ph.uniform();
                        sum += dust_density(*S, b.fracpos(x, y, z));
                    }
                } else {
                    for (int n = 0; n < Nrandom; n++) sum += dust_density(*S, rng.position(b));
                }
                mass[q - l] = sum/Nrandom*b.volume();            // TreeNodeSampleDensityCalculator.cpp:42-45
            };
            if (sampler == 1 && nthreads > 1) {
                std::atomic<size_t> next{l};
                auto worker = [&]() { size_t q; while ((q = next.fetch_add(1)) < lend) body(q); };
                vector<std::thread> th;
                for (int t = 1; t < nthreads; t++) th.emplace_back(worker);
                worker();
                for (auto& t : th) t.join();
            } else {
                for (size_t q = l; q < lend; q++) body(q);
            }
        }
        for (size_t q = l; q < lend; q++) {                          // TreeDustGrid.cpp:166-230
            bool need;
            if (lev <= minlevel) need = true;
            else if (lev < maxlevel) need = nocrit || mass[q - l]/total >= maxfrac;
            else need = false;
            if (need) T.split_node((int)q, type);
        }
        l = lend;
    }
    const int64_t n = (int64_t)T.box.size();
    *nnodes = n;
    delete S->grid; delete S;
    if (n > max_nodes) return SKG_ERR_CAPACITY;
    int m = 0;
    for (int64_t q = 0; q < n; q++) {
        const Box& b = T.box[q];
        box[6*q] = b.xmin; box[6*q+1] = b.ymin; box[6*q+2] = b.zmin;
        box[6*q+3] = b.xmax; box[6*q+4] = b.ymax; box[6*q+5] = b.zmax;
        split[q] = T.split[q]; child[q] = T.child[q]; father[q] = T.father[q]; dir[q] = T.dir[q];
        level[q] = T.level[q];
        cell[q] = T.child[q] < 0 ? m++ : -1;
    }
    return 0;
}


// The stellar emission phase for the packets [first, first+count) of every listed wavelength of a
// simulation of npp packets per wavelength (each carrying L_ell/npp), every packet drawing from its
// own counter-based stream keyed by (seed, packet id, wavelength): the tallies of any partition of
// [0, npp) into ranges sum to those of the whole range, up to the order of the FP64 additions --
// the reference's MPI task mode (MonteCarloSimulation.cpp:98-104) with a deterministic split.
// Needs scene->rho.
int orc_simulate_packets(const skg_scene* sc, uint64_t npp, uint64_t first, uint64_t count, int nthreads,
                         uint64_t seed, const int32_t* ells, int nell, double** cubes, double** seds,
                         double* labs_stel, orc_stats* st) {
    if (!sc->rho) { g_err = "orc_simulate_packets needs scene->rho"; return SKG_ERR_INVALID; }
    Sim* S = buildSim(sc);
    Sim& R = *S;
    const size_t nc = R.grid->ncells;
    R.rho.assign(sc->rho, sc->rho + nc*R.ncomp);
    vector<int> ellv;
    if (ells && nell > 0) ellv.assign(ells, ells + nell); else for (int e = 0; e < R.nlambda; e++) ellv.push_back(e);
    const uint64_t B = 1024, nblk = (count + B - 1)/B, nitems = ellv.size()*nblk;
    std::atomic<uint64_t> next{0};
    const auto t0 = std::chrono::steady_clock::now();
    auto worker = [&]() {
        Rng rng; rng.counter = true;
        Packet pp; Path path, ppath;
        uint64_t it;
        while ((it = next.fetch_add(1)) < nitems) {
            const int ell = ellv[it/nblk];
            const double L = R.Lv[ell]/npp;
            if (!(L > 0)) continue;
            const uint64_t b0 = first + (it % nblk)*B, b1 = std::min(first + count, b0 + B);
            for (uint64_t id = b0; id < b1; id++) {
                rng.ph = Philox(seed, id, 0xC0DE0000u + (uint32_t)ell);
                stellarLaunch(R, pp, ell, L, rng);
                R.stats.packets++;
                if (pp.L > 0) lifecycle(R, pp, path, ppath, rng, L/R.minWeightReduction, R.storeAbs, true);
            }
        }
    };
    vector<std::thread> th;
    for (int t = 1; t < nthreads; t++) th.emplace_back(worker);
    worker();
    for (auto& t : th) t.join();
    for (int i = 0; i < sc->ninstr; i++) {
        if (cubes && cubes[i] && !R.instr[i].cube.empty())
            std::memcpy(cubes[i], R.instr[i].cube.data(), R.instr[i].cube.size()*sizeof(double));
        if (seds && seds[i]) std::memcpy(seds[i], R.instr[i].sed.data(), R.instr[i].sed.size()*sizeof(double));
    }
    if (labs_stel) std::memcpy(labs_stel, R.LabsStel.data(), nc*R.nlambda*sizeof(double));
    if (st) {
        st->packets = R.stats.packets; st->steps = R.stats.steps; st->traversals = R.stats.traversals;
        st->scatterings = R.stats.scatterings; st->fallbacks = R.stats.fallbacks; st->npp = npp; st->chunks = nitems;
        st->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    delete R.grid; delete S;
    return 0;
}

// Runs a simulation: the stellar emission phase (MonteCarloSimulation::runstellaremission,
// MonteCarloSimulation.cpp:241-295) for `packages` per wavelength, optionally followed by
// `selfabs_cycles` dust self-absorption cycles (a fixed cycle count: at `packages` in one stage, or,
// with selfabs_staged, in each of the reference's three stages, PanMonteCarloSimulation.cpp:106-187)
// and the dust emission phase (:246-346).  If max_packets > 0 only that many
// packets of each phase run (a bounded sample for timing); Npp is unchanged so that the
// per-packet luminosity stays that of the full run.  st->seconds is the time of the packet loops
// of the phases (as the reference's TimeLogger times a phase), without the set-up.
// cubes[i]/seds[i] receive instrument i's tallies (layout of skg_read_instrument).
int orc_simulate(const skg_scene* sc, double packages, int nthreads, uint64_t seed, int selfabs_cycles,
                 int selfabs_staged, int dust_emission_phase, int64_t max_packets, const int32_t* ells, int nell,
                 double** cubes, double** seds,
                 double* labs_stel, double* labs_dust, double* temperature, orc_stats* st) {
    Sim* S = buildSim(sc);
    Sim& R = *S;
    size_t nc = R.grid->ncells;
    if (sc->rho) R.rho.assign(sc->rho, sc->rho + nc*R.ncomp);
    else if (R.ncomp) sampleDensity(R, sc->density_samples > 0 ? sc->density_samples : 100, nthreads, seed + 1000003);
    int nl = R.nlambda;
    // the stellar phase's wavelengths: all, or the given subset (a partial run of the same
    // simulation: each packet still carries L_ell/Npp)
    vector<int> ellv;
    if (ells && nell > 0) ellv.assign(ells, ells + nell); else for (int e = 0; e < nl; e++) ellv.push_back(e);
    const int nsel = (int)ellv.size();
    uint64_t Nchunks, chunksize, Npp;
    chunkParams(packages, nthreads, 1, nsel, Nchunks, chunksize, Npp);   // chunks over the wavelengths run
    std::atomic<int64_t> launched{0};
    double loop_seconds = 0;
    const auto t_loop = std::chrono::steady_clock::now();

    // stellar emission (MonteCarloSimulation.cpp:259-295)
    parallelCall(nthreads, (uint64_t)nsel*Nchunks, seed, [&](uint64_t index, Rng& rng) {
        int ell = ellv[index % nsel];
        double L = R.Lv[ell]/Npp;
        if (!(L > 0)) return;
        double Lthreshold = L/R.minWeightReduction;
        Packet pp; Path path, ppath;
        for (uint64_t i = 0; i < chunksize; i++) {
            if (max_packets > 0 && launched.fetch_add(1) >= max_packets) return;
            stellarLaunch(R, pp, ell, L, rng);
            R.stats.packets++;
            if (pp.L > 0) lifecycle(R, pp, path, ppath, rng, Lthreshold, R.storeAbs, true);
        }
    });
    loop_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t_loop).count();

    // dust self-absorption cycles and dust emission (PanMonteCarloSimulation.cpp:106-346)
    int dust_phases = 0;
    auto dustPhase = [&](double pk, bool selfabs) {
        const uint64_t phase_seed = seed + 7919*(uint64_t)(++dust_phases);
        calcDustEmission(R);
        if (selfabs) std::fill(R.LabsDust.begin(), R.LabsDust.end(), 0.0);   // rebootLabsdust
        uint64_t nch, csz, npp;
        chunkParams(pk, nthreads, 1, nl, nch, csz, npp);
        vector<vector<double>> cums(nl);
        vector<double> Ltots(nl), Lvs((size_t)nc*nl);
        for (int ell = 0; ell < nl; ell++) {
            vector<double> Lv(nc, 0.0);
            double Ltot = 0;
            for (size_t m = 0; m < nc; m++) {
                if (R.Labsbol[m] > 0.0) Lv[m] = R.Labsbol[m]*R.Lvv[m*nl + ell];
                Ltot += Lv[m];
            }
            Ltots[ell] = Ltot;
            if (Ltot > 0) cdf(cums[ell], Lv);
            for (size_t m = 0; m < nc; m++) Lvs[(size_t)ell*nc + m] = Lv[m];
        }
        std::atomic<int64_t> emitted{0};
        const auto t_dust = std::chrono::steady_clock::now();
        parallelCall(nthreads, (uint64_t)nl*nch, phase_seed, [&](uint64_t index, Rng& rng) {
            int ell = index % nl;
            double Ltot = Ltots[ell];
            if (!(Ltot > 0)) return;
            const vector<double>& Xv = cums[ell];
            Packet pp; Path path, ppath;
            double Lmean = Ltot/nc, Lem = Ltot/npp, Lth = Lem/R.minWeightReduction;
            double xi = R.dustEmissionBias;
            for (uint64_t i = 0; i < csz; i++) {
                if (max_packets > 0 && emitted.fetch_add(1) >= max_packets) return;
                int m; double weight = 1.0;
                double X = rng.uniform();
                if (selfabs) m = locate_clip(Xv.data(), nc+1, X);                 // :219-220
                else {                                                              // :306-322
                    if (X < xi) m = std::max(0, std::min((int)nc-1, static_cast<int>(nc*X/xi)));
                    else m = locate_clip(Xv.data(), nc+1, (X-xi)/(1-xi));
                    weight = 1.0/(1-xi+xi*Lmean/Lvs[(size_t)ell*nc + m]);
                }
                Vec r = R.grid->randomPositionInCell(m, rng);
                Vec k = rng.direction();
                pp = Packet{Lem*weight, ell, r, k, 0, -1};
                R.stats.packets++;
                lifecycle(R, pp, path, ppath, rng, Lth, selfabs, !selfabs);
            }
        });
        loop_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t_dust).count();
    };
    if (R.dustEmission && R.ncomp && !R.Tv.empty()) {
        if (selfabs_staged) {
            // rundustselfabsorption with a fixed cycle count (PanMonteCarloSimulation.cpp:106-187):
            // three stages of that many cycles with 1/10, 1/3 and 1 times the packages
            const double factor[3] = {1./10., 1./3., 1.};
            for (int stage = 0; stage < 3; stage++)
                for (int c = 0; c < selfabs_cycles; c++) dustPhase(packages*factor[stage], true);
        } else {
            for (int c = 0; c < selfabs_cycles; c++) dustPhase(packages, true);
        }
        if (dust_emission_phase) dustPhase(packages, false);
    }

    for (int i = 0; i < sc->ninstr; i++) {
        if (cubes && cubes[i] && !R.instr[i].cube.empty())
            std::memcpy(cubes[i], R.instr[i].cube.data(), R.instr[i].cube.size()*sizeof(double));
        if (seds && seds[i]) std::memcpy(seds[i], R.instr[i].sed.data(), R.instr[i].sed.size()*sizeof(double));
    }
    if (labs_stel) std::memcpy(labs_stel, R.LabsStel.data(), nc*nl*sizeof(double));
    if (labs_dust) std::memcpy(labs_dust, R.LabsDust.data(), nc*nl*sizeof(double));
    if (temperature && !R.Tcell.empty()) std::memcpy(temperature, R.Tcell.data(), nc*sizeof(double));
    if (st) {
        st->packets = R.stats.packets; st->steps = R.stats.steps; st->traversals = R.stats.traversals;
        st->scatterings = R.stats.scatterings; st->fallbacks = R.stats.fallbacks;
        st->npp = Npp; st->chunks = Nchunks;
        st->seconds = loop_seconds;
    }
    delete R.grid; delete S;
    return 0;
}

}  // extern "C"
