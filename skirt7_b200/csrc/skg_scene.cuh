// skg_scene.cuh -- device view of a simulation: dust mixes, stellar sources with their
// position samplers, instruments with their tallies, and the per-cell absorption tables.
#pragma once
#include "skg_grids.cuh"

namespace skg {

constexpr int MAX_STELLAR = 8;
constexpr int MAX_INSTR = 16;
constexpr int MAX_COMP = 4;

// Geometry with its launch sampler and density.
struct DevGeometry {
    int type;
    double p[6];
    // ExpDisk (ExpDiskGeometry.cpp:24-40)
    double hR, hz, Rmax, zmax, Rmin, rho0;
    // Sersic: 101-point tables s, S(s), M(s) (SersicFunction.cpp:17-76)
    const double* sv; const double* Sv; const double* Mv;
    double reff, srho0;
    // ClumpyGeometryDecorator (ClumpyGeometryDecorator.cpp:136-177)
    double f; int N; double h; int cutoff; int kernel;
    const double* clumps;     // 3*N, sorted on x
    const double* kXv;        // 401-point cubic spline cumulative mass (CubicSplineSmoothingKernel.cpp:22-38)
};

struct DevInstr {
    int type;
    double costheta, sintheta, cosphi, sinphi, cospa, sinpa;
    double kx, ky, kz;        // direction towards the observer (DistantInstrument.cpp:43)
    int nxp, nyp;
    double xpmin, ypmin, xpsiz, ypsiz;
    int nscatt_levels;
    int ncomp;                // tally components (1, or SKG_FULL_NBASE + levels)
    double* cube;             // [ncomp][nlambda][nyp*nxp]
    double* sed;              // [ncomp][nlambda]
};

struct DevScene {
    int nlambda;
    const double* lambda;
    const double* dlambda;
    int ncomp;
    const double* kext;       // [h*nl + ell]
    const double* ksca;
    const double* albedo;
    const double* asym;
    const double* rho;        // [h*ncells + m]
    const float*  rhof;
    int ncells;

    int nstellar;
    DevGeometry stellar[MAX_STELLAR];
    const double* starL;      // [h*nl + ell]
    const double* Lv;         // [ell]
    const double* Xvv;        // [ell*(nstellar+1) + h]
    double emission_bias;

    int ninstr;
    DevInstr instr[MAX_INSTR];
    int ngroups;
    int group_start[MAX_INSTR + 1];   // instruments of group q: group_instr[group_start[q] .. group_start[q+1])
    int group_instr[MAX_INSTR];
    int group_frame_only[MAX_INSTR];  // all members are Frame instruments (pixel test before traversal)
    double gkx[MAX_INSTR], gky[MAX_INSTR], gkz[MAX_INSTR];
    int sed_base[MAX_INSTR];          // offset of each instrument's SED bins in a concatenation
    int sed_bins;                     // SED bins of all instruments

    double min_weight_reduction;
    int min_scatt_events;
    double xi;
    int store_abs;
    double* labs_stel;        // [ell*ncells + m] (wavelength-major on the device)
    double* labs_dust;

    // dust emission sources
    const double* emit_cdf;   // [ell][ncells+1] normalised cumulative luminosity per wavelength
    const double* emit_Ltot;  // [ell]
    const double* emit_Lv;    // [ell][ncells] cell luminosity (emission bias weights)
    double dust_emission_bias;
};

// One launch carries slices of one or more simulations ("slots").  A work item is one slice: the
// packets [first, first+count) of every listed wavelength of the simulation in `slot`, each with
// luminosity L/npp_total.  Global packet index p belongs to the item with begin <= p < begin +
// count*nell.  The header and the tables live in device memory so that a captured launch can be
// replayed with new contents.
struct WorkItem {
    int slot;
    int nell;
    int ell0;                 // wavelengths: ells[ell0 .. ell0 + nell)
    int pad;
    uint64_t npp_total;
    uint64_t first, count;
    uint64_t seed;
    uint64_t begin;
};
struct BatchHeader {
    int phase;
    int nslots;
    int nitems;
    int pad;
    uint64_t total;           // packets of all items
};
constexpr int MAX_SLOTS = 64;

struct RunParams {
    const BatchHeader* hdr;
    const WorkItem* items;
    const DevGrid* grids;         // [nslots]
    const DevScene* const* scenes; // [nslots]
    const int* ells;
    int max_scatt;
    int refill;                   // lanes of a warp that wait for a job before it takes new ones (0: default)
    unsigned long long* work;     // packet work counter
    unsigned int* err;            // error word
    unsigned long long* counters; // skg_counters layout
};

// ---------------------------------------------------------------------------------------------
// Wavefront state.  The packets in flight live in a pool of 128-byte records; each wave an event
// pass (one thread per record) advances every packet to its next traversals and writes them as
// jobs, and a traversal pass walks all jobs of the wave.
enum PacketState : int { PK_EMPTY = 0, PK_WAIT, PK_INTERACT, PK_TERM, PK_DONE };
constexpr int JOB_MAIN = 31;          // job type of the packet's own path; 0..15 = peel-off group

struct __align__(16) Packet {
    double x, y, z;                   // position (rounded to the traversal precision)
    double kx, ky, kz;                // direction
    double L, Lth;                    // luminosity and its termination threshold
    double s_int;                     // distance to the interaction point (result of the path job)
    uint64_t id;                      // packet number within its work item (RNG counter words)
    int item;                         // work item
    int ell;
    int nscatt;
    int pos_cell;                     // cell of the position: -2 unknown, -1 outside the grid
    int int_cell;                     // cell of the interaction point (-1 unknown)
    unsigned rngc;                    // next Philox block of the packet's stream
    int state;                        // PacketState
    int flags;                        // bit 0 stellar origin, bit 1 the pending peel-offs follow a scattering
    int peel_j0, peel_n;              // this packet's peel-off jobs of the last wave
    int pad[2];
};
static_assert(sizeof(Packet) == 128, "packet record is two 64-byte lines");

struct WaveParams {
    RunParams R;
    Packet* pk;
    int npool;
    int wave;                         // index of this wave within the phase
    // this wave's jobs (written by the event pass, walked by the traversal pass): path jobs at
    // [0, npool) and peel-off jobs from npool on, so that the longest jobs are taken first
    int2* jobs;                       // (packet, type)
    double* jtau;                     // peel-off optical depth
    double* jL;                       // peel-off luminosity
    unsigned* jcount;                 // [0] path jobs, [1] peel-off jobs, [2] jobs taken by the
                                      // traversal pass (its path kernel when split), [3] packets
                                      // with jobs, [4] peel-off jobs taken by a split pass,
                                      // [5] records on the free list, [6] on the interaction list
    // the previous wave's jobs (peel-off detection)
    const int2* pjobs;
    const double* pjtau;
    const double* pjL;
    unsigned* last_busy;              // highest wave index that had jobs
    int* freelist;                    // records the event pass freed (count: jcount[5])
    int* intlist;                     // records it found at their interaction point (jcount[6])
    float4* ckpt;                     // per packet record: checkpoints of its path walk
    // the grid of a single-simulation launch: the traversal kernels' instantiation for one slot
    // reads it from their parameters (constant-bank operands, no load instructions per cell step)
    DevGrid g0;
};

// ---------------------------------------------------------------------------------------------
// samplers

// Lambert W, branch -1, on [-1/e, 0) (the function SpecialFunctions::LambertW1 evaluates,
// SKIRTcore/SpecialFunctions.cpp:579): Halley iteration from the branch-point series in
// p = -sqrt(2(1+ez)) or from the asymptotic log form.
SKG_D double lambert_w1(double z) {
    if (z == 0.0) return -DBL_MAX;
    const double em1 = 0.36787944117144233;
    double q = z + em1;
    double w;
    if (q < 0.3) {
        double p = -sqrt(2.0 * 2.718281828459045 * fmax(q, 0.0));
        w = -1.0 + p - p * p / 3.0 + 11.0 / 72.0 * p * p * p - 43.0 / 540.0 * p * p * p * p;
    } else {
        double l1 = log(-z), l2 = log(-l1);
        w = l1 - l2 + l2 / l1;
    }
    if (q < 1e-12) return w;
    for (int i = 0; i < 50; i++) {
        double e = exp(w), f = w * e - z, wp1 = w + 1.0;
        if (wp1 == 0.0) break;
        double dw = f / (e * wp1 - (w + 2.0) * f / (2.0 * wp1));
        w -= dw;
        if (fabs(dw) <= 1e-15 * fabs(w)) break;
    }
    return w;
}

// isotropic direction (Random::direction, Random.cpp:180-185, Direction.cpp:12-38)
SKG_D V3<double> iso_direction(Philox& rng) {
    double theta = acos(2.0 * rng.uniform() - 1.0);
    double phi = 2.0 * M_PI * rng.uniform();
    if (theta <= 1e-8) return mk3(0.0, 0.0, 1.0);
    if (theta >= M_PI - 1e-8) return mk3(0.0, 0.0, -1.0);
    double st = sin(theta), sp, cp;
    sincos(phi, &sp, &cp);
    return mk3(st * cp, st * sp, cos(theta));
}

// NR::locate_clip on a device table (NR.hpp:145-151)
SKG_D int dlocate_clip(const double* xv, int size, double x) {
    if (x < xv[0]) return 0;
    int jl = -1, ju = size - 1;
    while (ju - jl > 1) { int jm = (ju + jl) >> 1; if (x < xv[jm]) ju = jm; else jl = jm; }
    return jl;
}
SKG_D double interp_loglog(double x, double x1, double x2, double f1, double f2) {   // NR.hpp:318-345
    x = log10(x); x1 = log10(x1); x2 = log10(x2);
    bool logf = f1 > 0 && f2 > 0;
    if (logf) { f1 = log10(f1); f2 = log10(f2); }
    double fx = f1 + ((x - x1) / (x2 - x1)) * (f2 - f1);
    if (logf) fx = pow(10.0, fx);
    return fx;
}

SKG_D double sersic_S(const DevGeometry& G, double s) {          // SersicFunction.cpp:80-92
    if (s <= G.sv[0]) return G.Sv[0];
    if (s >= G.sv[100]) return G.Sv[100];
    int i = dlocate_clip(G.sv, 101, s);
    return interp_loglog(s, G.sv[i], G.sv[i + 1], G.Sv[i], G.Sv[i + 1]);
}

SKG_D double geom_base_density(const DevGeometry& G, double x, double y, double z) {
    if (G.type == 0) {                                              // ExpDiskGeometry.cpp:117-129
        double R = sqrt(x * x + y * y), az = fabs(z);
        if (G.Rmax > 0.0 && R > G.Rmax) return 0.0;
        if (G.zmax > 0.0 && az > G.zmax) return 0.0;
        if (R < G.Rmin) return 0.0;
        return G.rho0 * exp(-R / G.hR) * exp(-az / G.hz);
    } else if (G.type == 1) {                                       // SersicGeometry.cpp:72-77
        return G.srho0 * sersic_S(G, sqrt(x * x + y * y + z * z) / G.reff);
    } else if (G.type == 3) {
        double c = G.p[0], u2 = (x * x + y * y + z * z) / (c * c);
        return 3.0 / (4.0 * M_PI * c * c * c) * pow(1.0 + u2, -2.5);
    }
    return (x == 0 && y == 0 && z == 0) ? INFINITY : 0.0;            // PointGeometry.cpp:27-32
}

SKG_D double kernel_density(int kernel, double u) {
    if (u < 0.0 || u > 1.0) return 0.0;
    if (kernel == 1) return 0.75 / M_PI;                             // UniformSmoothingKernel
    if (u < 0.5) return 8.0 / M_PI * (1.0 - 6.0 * u * u * (1.0 - u));  // CubicSplineSmoothingKernel.cpp:42-50
    return 8.0 / M_PI * 2.0 * (1.0 - u) * (1.0 - u) * (1.0 - u);
}

// NR::locate on the x-sorted clump list (as ClumpyGeometryDecorator::density uses it)
SKG_D int locate_clump(const DevGeometry& G, double x) {
    int n = G.N;
    if (x < G.clumps[0]) return -1;
    if (G.clumps[3 * (n - 1)] < x) return n - 1;
    int jl = -1, ju = n;
    while (ju - jl > 1) { int jm = (ju + jl) >> 1; if (x < G.clumps[3 * jm]) ju = jm; else jl = jm; }
    if (jl <= 0) return 0;
    if (jl >= n - 2) return n - 2;
    return jl;
}

SKG_D double geom_density(const DevGeometry& G, double x, double y, double z) {
    if (G.N == 0) return geom_base_density(G, x, y, z);
    double rhosmooth = (1.0 - G.f) * geom_base_density(G, x, y, z);   // ClumpyGeometryDecorator.cpp:136-154
    if (G.cutoff && !rhosmooth) return 0.0;
    double rhoc = 0.0, Mclump = G.f / G.N, h3 = G.h * G.h * G.h;
    int i0 = max(0, locate_clump(G, x - G.h));
    int i1 = max(0, locate_clump(G, x + G.h));
    for (int i = i0; i <= i1; i++) {
        double dx = x - G.clumps[3 * i], dy = y - G.clumps[3 * i + 1], dz = z - G.clumps[3 * i + 2];
        double u = sqrt(dx * dx + dy * dy + dz * dz) / G.h;
        rhoc += Mclump * kernel_density(G.kernel, u) / h3;
    }
    return rhosmooth + rhoc;
}

SKG_D V3<double> geom_base_position(const DevGeometry& G, Philox& rng) {
    if (G.type == 0) {                                               // SepAxGeometry.cpp:20-30
        double R, X;
        int guard = 0;
        do {                                                         // ExpDiskGeometry.cpp:133-144
            X = rng.uniform();
            R = G.hR * (-1.0 - lambert_w1((X - 1.0) / 2.718281828459045));
        } while (((G.Rmax > 0.0 && R >= G.Rmax) || R <= G.Rmin) && ++guard < 1000);
        double phi = 2.0 * M_PI * rng.uniform();
        double z;
        guard = 0;
        do {                                                         // ExpDiskGeometry.cpp:148-161
            X = rng.uniform();
            z = (X <= 0.5) ? G.hz * log(2.0 * X) : -G.hz * log(2.0 * (1.0 - X));
        } while (G.zmax > 0.0 && fabs(z) >= G.zmax && ++guard < 1000);
        double sp, cp; sincos(phi, &sp, &cp);
        return mk3(R * cp, R * sp, z);
    } else if (G.type == 1 || G.type == 3) {                         // SpheGeometry.cpp:36-44
        double r;
        double X = rng.uniform();
        if (G.type == 1) {                                           // SersicGeometry.cpp:84-90
            if (X <= G.Mv[0]) r = G.sv[0];
            else if (X >= G.Mv[100]) r = G.sv[100];
            else { int i = dlocate_clip(G.Mv, 101, X); r = interp_loglog(X, G.Mv[i], G.Mv[i + 1], G.sv[i], G.sv[i + 1]); }
            r *= G.reff;
        } else {
            r = G.p[0] / sqrt(pow(X, -2.0 / 3.0) - 1.0);
        }
        V3<double> k = iso_direction(rng);
        return mk3(r * k.x, r * k.y, r * k.z);
    }
    return mk3(0.0, 0.0, 0.0);
}

SKG_D double kernel_radius(const DevGeometry& G, Philox& rng) {
    double X = rng.uniform();
    if (G.kernel == 1) return cbrt(X);                               // UniformSmoothingKernel
    int k = dlocate_clip(G.kXv, 401, X);                              // CubicSplineSmoothingKernel.cpp:54-61
    double p = (X - G.kXv[k]) / (G.kXv[k + 1] - G.kXv[k]);
    return (k + p) / 400.0;
}

SKG_D V3<double> geom_position(const DevGeometry& G, Philox& rng) {
    if (G.N == 0) return geom_base_position(G, rng);
    for (int guard = 0; guard < 10000; guard++) {                     // ClumpyGeometryDecorator.cpp:158-177
        double X = rng.uniform();
        if (X > G.f) return geom_base_position(G, rng);
        int i = min((int)((X / G.f) * G.N), G.N - 1);
        double u = kernel_radius(G, rng);
        V3<double> k = iso_direction(rng);
        double x = G.clumps[3 * i] + u * G.h * k.x, y = G.clumps[3 * i + 1] + u * G.h * k.y,
               z = G.clumps[3 * i + 2] + u * G.h * k.z;
        if (!G.cutoff || geom_base_density(G, x, y, z)) return mk3(x, y, z);
    }
    return geom_base_position(G, rng);
}

// SingleFrameInstrument::pixelondetector (SingleFrameInstrument.cpp:130-147)
SKG_D int pixel_on_detector(const DevInstr& I, double x, double y, double z) {
    double xpp = -I.sinphi * x + I.cosphi * y;
    double ypp = -I.cosphi * I.costheta * x - I.sinphi * I.costheta * y + I.sintheta * z;
    double xp = I.cospa * xpp - I.sinpa * ypp;
    double yp = I.sinpa * xpp + I.cospa * ypp;
    double fi = floor((xp - I.xpmin) / I.xpsiz);
    double fj = floor((yp - I.ypmin) / I.ypsiz);
    // a non-finite position maps off the detector (the x86 conversion of NaN gives INT_MIN there)
    if (!(fi >= 0.0 && fi < (double)I.nxp && fj >= 0.0 && fj < (double)I.nyp)) return -1;
    return (int)fi + I.nxp * (int)fj;
}

// Random position in cell m (DustGrid::randomPositionInCell).
SKG_D V3<double> random_position_in_cell(const DevGrid& g, int m, Philox& rng) {
    double lx, ly, lz, hx, hy, hz;
    if (g.type == SKG_GRID_CARTESIAN) {                       // CartesianDustGrid.cpp:333-343
        int i = m / (g.nz * g.ny), j = (m / g.nz) % g.ny, k = m % g.nz;
        lx = g.xv[i]; ly = g.yv[j]; lz = g.zv[k]; hx = g.xv[i + 1]; hy = g.yv[j + 1]; hz = g.zv[k + 1];
    } else if (g.type == SKG_GRID_VORONOI) {                  // VoronoiMesh.cpp:620-648
        const double* b = g.vbbox + 6 * (size_t)m;
        const double* pm = g.site + 3 * (size_t)m;
        for (int it = 0; it < 10000; it++) {
            double x = rng.uniform(), y = rng.uniform(), z = rng.uniform();
            x = b[0] + x * (b[3] - b[0]); y = b[1] + y * (b[4] - b[1]); z = b[2] + z * (b[5] - b[2]);
            double dx = x - pm[0], dy = y - pm[1], dz = z - pm[2];
            double target = dx * dx + dy * dy + dz * dz;
            bool ok = true;
            for (int q = g.vnoff[m]; q < g.vnoff[m + 1]; q++) {
                int id = g.vnbr[q];
                if (id < 0) continue;
                const double* pi = g.site + 3 * (size_t)id;
                double ex = x - pi[0], ey = y - pi[1], ez = z - pi[2];
                if (ex * ex + ey * ey + ez * ez < target) { ok = false; break; }
            }
            if (ok) return mk3(x, y, z);
        }
        return mk3(pm[0], pm[1], pm[2]);
    } else {                                                   // TreeDustGrid.cpp:366-369
        const double* b = g.node_box + 6 * (size_t)g.cell_node[m];
        lx = b[0]; ly = b[1]; lz = b[2]; hx = b[3]; hy = b[4]; hz = b[5];
    }
    double x = rng.uniform(), y = rng.uniform(), z = rng.uniform();   // Random.cpp:227-235
    return mk3(lx + x * (hx - lx), ly + y * (hy - ly), lz + z * (hz - lz));
}

// Random::direction(bfk, costheta) (Random.cpp:189-223)
SKG_D V3<double> rotate_direction(V3<double> k, double costheta, Philox& rng) {
    double phi = 2.0 * M_PI * rng.uniform();
    double sinphi, cosphi; sincos(phi, &sinphi, &cosphi);
    double sintheta = sqrt(fabs((1.0 - costheta) * (1.0 + costheta)));
    if (k.z > 0.99999) return mk3(cosphi * sintheta, sinphi * sintheta, costheta);
    if (k.z < -0.99999) return mk3(cosphi * sintheta, sinphi * sintheta, -costheta);
    double root = sqrt((1.0 - k.z) * (1.0 + k.z));
    return mk3(sintheta / root * (-k.x * k.z * cosphi + k.y * sinphi) + k.x * costheta,
               -sintheta / root * (k.y * k.z * cosphi + k.x * sinphi) + k.y * costheta,
               root * sintheta * cosphi + k.z * costheta);
}

}  // namespace skg
