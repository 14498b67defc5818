// skg_voronoi.cu -- Voronoi tessellation of the dust grid sites on the device
// (the product of VoronoiMesh::buildMesh, VoronoiMesh.cpp:297-405, which uses Voro++).
//
// Each thread builds one cell by clipping the domain box with the bisector planes of nearby
// sites.  The convex cell is held in its dual form: every polyhedron vertex is a triangle of
// the three planes meeting there, stored with a consistent orientation.  Clipping by a plane
// removes the triangles whose vertex lies outside it and closes the hole with one new triangle
// (x, y, P) per boundary edge x->y -- the boundary needs no explicit ordering.  Candidate sites
// come from a uniform bin grid, visited in growing shells (sorted by distance within a shell)
// until no unvisited site can be closer than twice the cell's current radius (the security
// radius), after which no further plane can cut the cell.  Coordinates are relative to the site.
//
// Outputs per cell: neighbour ids (walls -1..-6 as Voro++ numbers them), volume, centroid and
// bounding box; the host adds the nb^3 block lists of VoronoiMesh.cpp:334-404.
#include "skg_scene.cuh"
#include "skg_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <type_traits>
#include <vector>

using namespace skg;

namespace {

// capacities of the device construction (a cell that exceeds one is rebuilt on the host with
// the larger ones below)
constexpr int VMAXP = 112;     // clipping planes per cell (6 walls included)
constexpr int VMAXT = 224;     // dual triangles (polyhedron vertices)
constexpr int VMAXC = 96;      // candidates per shell
constexpr int VMAXN = 80;      // neighbours stored per cell
constexpr int HMAXP = 1024, HMAXT = 2048, HMAXC = 512, HMAXN = 1000;

struct BinGrid {
    double lo[3], h[3];
    int n[3];
    const int* off;     // n0*n1*n2 + 1
    const int* ids;
};

struct Plane { double x, y, z, d; };

template<typename I>
__host__ __device__ __forceinline__ void tri_vertex(const Plane* P, const I* t, double* v) {
    const Plane &a = P[t[0]], &b = P[t[1]], &c = P[t[2]];
    // Cramer: v = (d_a (b x c) + d_b (c x a) + d_c (a x b)) / (a . (b x c))
    double bcx = b.y * c.z - b.z * c.y, bcy = b.z * c.x - b.x * c.z, bcz = b.x * c.y - b.y * c.x;
    double cax = c.y * a.z - c.z * a.y, cay = c.z * a.x - c.x * a.z, caz = c.x * a.y - c.y * a.x;
    double abx = a.y * b.z - a.z * b.y, aby = a.z * b.x - a.x * b.z, abz = a.x * b.y - a.y * b.x;
    double det = a.x * bcx + a.y * bcy + a.z * bcz;
    double inv = 1.0 / det;
    v[0] = (a.d * bcx + b.d * cax + c.d * abx) * inv;
    v[1] = (a.d * bcy + b.d * cay + c.d * aby) * inv;
    v[2] = (a.d * bcz + b.d * caz + c.d * abz) * inv;
}

// Builds the cell of site i with capacities MP planes, MT polyhedron vertices, MC candidates per
// batch and MN stored neighbours, writing its results to output slot o; callable on the host too
// (the rebuild of cells that exceed the device capacities).
template<int MP, int MT, int MC, int MN>
__host__ __device__ void voronoi_cell_t(int i, int o, const double* __restrict__ sites, const double* __restrict__ ext,
                                        const BinGrid& G, int* nbr_count, int* nbr_ids, double* volume,
                                        double* centroid, double* bbox, int* status) {
    using PIdx = typename std::conditional<(MP <= 255), unsigned char, unsigned short>::type;
    const double px = sites[3 * i], py = sites[3 * i + 1], pz = sites[3 * i + 2];

    Plane P[MP];
    int pid[MP];
    PIdx T[MT][3];
    double V[MT][3];
    int np = 6, nt = 0;
    int st = 0;

    // walls: outward normals, relative to the site; ids -1..-6 = xmin,xmax,ymin,ymax,zmin,zmax
    P[0] = {-1, 0, 0, -(ext[0] - px)}; pid[0] = -1;
    P[1] = {1, 0, 0, ext[3] - px};     pid[1] = -2;
    P[2] = {0, -1, 0, -(ext[1] - py)}; pid[2] = -3;
    P[3] = {0, 1, 0, ext[4] - py};     pid[3] = -4;
    P[4] = {0, 0, -1, -(ext[2] - pz)}; pid[4] = -5;
    P[5] = {0, 0, 1, ext[5] - pz};     pid[5] = -6;
    for (int c = 0; c < 8; c++) {
        PIdx a = (c & 1) ? 1 : 0, b = (c & 2) ? 3 : 2, d = (c & 4) ? 5 : 4;
        // orientation: det(n_a, n_b, n_d) > 0
        double s = P[a].x * (P[b].y * P[d].z - P[b].z * P[d].y) - P[a].y * (P[b].x * P[d].z - P[b].z * P[d].x)
                 + P[a].z * (P[b].x * P[d].y - P[b].y * P[d].x);
        if (s > 0) { T[nt][0] = a; T[nt][1] = b; T[nt][2] = d; }
        else       { T[nt][0] = a; T[nt][1] = d; T[nt][2] = b; }
        tri_vertex(P, T[nt], V[nt]);
        nt++;
    }
    double R2 = 0;
    for (int t = 0; t < nt; t++) R2 = fmax(R2, V[t][0] * V[t][0] + V[t][1] * V[t][1] + V[t][2] * V[t][2]);

    int b0 = max(0, min(G.n[0] - 1, (int)((px - G.lo[0]) / G.h[0])));
    int b1 = max(0, min(G.n[1] - 1, (int)((py - G.lo[1]) / G.h[1])));
    int b2 = max(0, min(G.n[2] - 1, (int)((pz - G.lo[2]) / G.h[2])));
    int maxs = max(G.n[0], max(G.n[1], G.n[2]));
    int cand[MC];
    double cd2[MC];
    bool outside[MT];

    for (int s = 0; s <= maxs && !st; s++) {
        // smallest distance from the site to any bin at Chebyshev distance >= s
        if (s > 0) {
            double dmin = 1e300;
            double lo0 = G.lo[0] + (b0 - s + 1) * G.h[0], hi0 = G.lo[0] + (b0 + s) * G.h[0];
            double lo1 = G.lo[1] + (b1 - s + 1) * G.h[1], hi1 = G.lo[1] + (b1 + s) * G.h[1];
            double lo2 = G.lo[2] + (b2 - s + 1) * G.h[2], hi2 = G.lo[2] + (b2 + s) * G.h[2];
            if (b0 - s >= 0) dmin = fmin(dmin, px - lo0);
            if (b0 + s < G.n[0]) dmin = fmin(dmin, hi0 - px);
            if (b1 - s >= 0) dmin = fmin(dmin, py - lo1);
            if (b1 + s < G.n[1]) dmin = fmin(dmin, hi1 - py);
            if (b2 - s >= 0) dmin = fmin(dmin, pz - lo2);
            if (b2 + s < G.n[2]) dmin = fmin(dmin, hi2 - pz);
            if (dmin >= 1e300) break;                       // every bin visited
            if (dmin > 0 && dmin * dmin > 4.0 * R2) break;  // security radius reached
        }
        // gather the shell's candidates, nearest first; a full list is clipped and emptied
        int nc = 0;
        bool shell_done = false;
        int x = b0 - s, y = b1 - s, z = b2 - s - 1;
        int q = 0, q1 = 0;
        while (!st) {
          bool have = false;
          int jnext = -1; double d2next = 0;
          while (!have) {
            if (q < q1) {
                int j = G.ids[q++];
                if (j == i) continue;
                double dx = sites[3 * j] - px, dy = sites[3 * j + 1] - py, dz = sites[3 * j + 2] - pz;
                double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 >= 4.0 * R2) continue;
                jnext = j; d2next = d2; have = true;
                break;
            }
            // next bin of the shell
            if (++z > b2 + s) { z = b2 - s; if (++y > b1 + s) { y = b1 - s; if (++x > b0 + s) { shell_done = true; break; } } }
            if (x < 0 || x >= G.n[0] || y < 0 || y >= G.n[1] || z < 0 || z >= G.n[2]) continue;
            if (max(abs(x - b0), max(abs(y - b1), abs(z - b2))) != s) continue;
            int bin = (x * G.n[1] + y) * G.n[2] + z;
            q = G.off[bin]; q1 = G.off[bin + 1];
          }
          if (have) {
            int k = nc++;
            while (k > 0 && cd2[k - 1] > d2next) { cd2[k] = cd2[k - 1]; cand[k] = cand[k - 1]; k--; }
            cd2[k] = d2next; cand[k] = jnext;
            if (nc < MC) continue;
          }
          // clip by the collected candidates, nearest first
          for (int c = 0; c < nc && !st; c++) {
            if (cd2[c] >= 4.0 * R2) break;
            int j = cand[c];
            double nx = sites[3 * j] - px, ny = sites[3 * j + 1] - py, nz = sites[3 * j + 2] - pz;
            double d = 0.5 * (nx * nx + ny * ny + nz * nz);
            int nout = 0;
            for (int t = 0; t < nt; t++) {
                outside[t] = nx * V[t][0] + ny * V[t][1] + nz * V[t][2] > d;
                nout += outside[t];
            }
            if (nout == 0) continue;
            if (nout == nt || np >= MP) { st = 2; break; }
            int pnew = np;
            P[np] = {nx, ny, nz, d}; pid[np] = j; np++;
            // new triangles on the boundary of the removed region
            int nnew = 0;
            PIdx NT[MT][3];
            for (int t = 0; t < nt && !st; t++) {
                if (!outside[t]) continue;
                for (int e = 0; e < 3; e++) {
                    PIdx x = T[t][e], y = T[t][(e + 1) % 3];
                    // the triangle across edge x->y holds y->x
                    int u = -1;
                    for (int w = 0; w < nt; w++) {
                        if (w == t) continue;
                        const PIdx* W = T[w];
                        if ((W[0] == y && W[1] == x) || (W[1] == y && W[2] == x) || (W[2] == y && W[0] == x)) { u = w; break; }
                    }
                    if (u < 0) { st = 3; break; }
                    if (!outside[u]) {
                        if (nnew >= MT) { st = 1; break; }
                        NT[nnew][0] = x; NT[nnew][1] = y; NT[nnew][2] = (PIdx)pnew; nnew++;
                    }
                }
            }
            if (st) break;
            int w = 0;
            for (int t = 0; t < nt; t++) {
                if (outside[t]) continue;
                if (w != t) { T[w][0] = T[t][0]; T[w][1] = T[t][1]; T[w][2] = T[t][2];
                              V[w][0] = V[t][0]; V[w][1] = V[t][1]; V[w][2] = V[t][2]; }
                w++;
            }
            if (w + nnew > MT) { st = 1; break; }
            for (int q = 0; q < nnew; q++) {
                T[w][0] = NT[q][0]; T[w][1] = NT[q][1]; T[w][2] = NT[q][2];
                tri_vertex(P, T[w], V[w]);
                w++;
            }
            nt = w;
            R2 = 0;
            for (int t = 0; t < nt; t++) R2 = fmax(R2, V[t][0] * V[t][0] + V[t][1] * V[t][1] + V[t][2] * V[t][2]);
          }
          nc = 0;
          if (shell_done) break;
        }
    }

    // neighbours: planes that still bound the cell, volume and centroid by walking each face
    int nn = 0;
    double vol = 0, cx = 0, cy = 0, cz = 0;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int t = 0; t < nt; t++)
        for (int c = 0; c < 3; c++) { lo[c] = fmin(lo[c], V[t][c]); hi[c] = fmax(hi[c], V[t][c]); }
    for (int p = 0; p < np && !st; p++) {
        int t0 = -1, k0 = 0;
        for (int t = 0; t < nt && t0 < 0; t++)
            for (int c = 0; c < 3; c++) if (T[t][c] == p) { t0 = t; k0 = c; break; }
        if (t0 < 0) continue;
        if (nn >= MN) { st = 1; break; }
        nbr_ids[(size_t)o * MN + nn++] = pid[p];
        // walk around plane p: triangle (p, a, b) -> the triangle holding p followed by b
        int t = t0, k = k0, guard = 0;
        const double* A0 = V[t0];
        const double* prev = nullptr;
        do {
            PIdx b = T[t][(k + 2) % 3];
            const double* cur = V[t];
            if (prev) {
                // tetrahedron (site, A0, prev, cur)
                double d6 = A0[0] * (prev[1] * cur[2] - prev[2] * cur[1]) - A0[1] * (prev[0] * cur[2] - prev[2] * cur[0])
                          + A0[2] * (prev[0] * cur[1] - prev[1] * cur[0]);
                vol += d6;
                cx += d6 * (A0[0] + prev[0] + cur[0]); cy += d6 * (A0[1] + prev[1] + cur[1]); cz += d6 * (A0[2] + prev[2] + cur[2]);
            }
            prev = cur;
            int nxt = -1, nk = 0;
            for (int w = 0; w < nt && nxt < 0; w++)
                for (int c = 0; c < 3; c++) if (T[w][c] == p && T[w][(c + 1) % 3] == b) { nxt = w; nk = c; break; }
            if (nxt < 0) { st = 3; break; }
            t = nxt; k = nk;
        } while (t != t0 && ++guard < MT);
        if (guard >= MT) st = 3;
    }
    nbr_count[o] = nn;
    double V6 = vol;
    volume[o] = fabs(V6) / 6.0;
    if (V6 != 0) { centroid[3 * o] = px + cx / (4.0 * V6); centroid[3 * o + 1] = py + cy / (4.0 * V6); centroid[3 * o + 2] = pz + cz / (4.0 * V6); }
    else { centroid[3 * o] = px; centroid[3 * o + 1] = py; centroid[3 * o + 2] = pz; }
    bbox[6 * o] = px + lo[0]; bbox[6 * o + 1] = py + lo[1]; bbox[6 * o + 2] = pz + lo[2];
    bbox[6 * o + 3] = px + hi[0]; bbox[6 * o + 4] = py + hi[1]; bbox[6 * o + 5] = pz + hi[2];
    status[o] = st;
}

__global__ void voronoi_cell_kernel(const double* __restrict__ sites, int nsites, const double* __restrict__ ext,
                                    BinGrid G, int* nbr_count, int* nbr_ids, double* volume, double* centroid,
                                    double* bbox, int* status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsites) return;
    voronoi_cell_t<VMAXP, VMAXT, VMAXC, VMAXN>(i, i, sites, ext, G, nbr_count, nbr_ids, volume, centroid, bbox, status);
}

}  // namespace

struct skg_voronoi {
    double ext[6];
    std::vector<double> sites;            // kept sites (3 per cell)
    std::vector<int64_t> noff;
    std::vector<int32_t> nbr;
    std::vector<double> volume, centroid, bbox;
    int nb = 0;
    std::vector<int64_t> boff;
    std::vector<int32_t> bids;
};

extern "C" {

int skg_voronoi_build(const double* sites, int32_t nsites, double xmin, double ymin, double zmin, double xmax,
                      double ymax, double zmax, int device, skg_voronoi** out) {
    *out = nullptr;
    if (!sites || nsites <= 0 || !(xmax > xmin && ymax > ymin && zmax > zmin)) {
        set_error("Voronoi construction needs sites and a non-empty extent");
        return SKG_ERR_INVALID;
    }
    skg_voronoi* v = new skg_voronoi();
    double ext[6] = {xmin, ymin, zmin, xmax, ymax, zmax};
    std::memcpy(v->ext, ext, sizeof(ext));
    double dx = xmax - xmin, dy = ymax - ymin, dz = zmax - zmin;
    double eps = 1e-12 * std::sqrt(dx * dx + dy * dy + dz * dz);     // VoronoiMesh.cpp:220
    // keep the sites inside the extent and drop those closer than eps to a later one in x order
    // (VoronoiMesh::buildMesh with removeNearby, VoronoiMesh.cpp:300-325)
    std::vector<int> idx;
    for (int m = 0; m < nsites; m++) {
        const double* p = sites + 3 * (size_t)m;
        if (p[0] >= xmin && p[0] <= xmax && p[1] >= ymin && p[1] <= ymax && p[2] >= zmin && p[2] <= zmax) idx.push_back(m);
    }
    std::vector<int> order(idx);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return sites[3 * (size_t)a] < sites[3 * (size_t)b]; });
    std::vector<char> drop(nsites, 0);
    for (size_t i = 0; i < order.size(); i++) {
        const double* pi = sites + 3 * (size_t)order[i];
        for (size_t j = i + 1; j < order.size() && sites[3 * (size_t)order[j]] - pi[0] < eps; j++) {
            const double* pj = sites + 3 * (size_t)order[j];
            double ex = pj[0] - pi[0], ey = pj[1] - pi[1], ez = pj[2] - pi[2];
            if (ex * ex + ey * ey + ez * ez < eps * eps) { drop[order[i]] = 1; break; }
        }
    }
    for (int m : idx) if (!drop[m]) v->sites.insert(v->sites.end(), sites + 3 * (size_t)m, sites + 3 * (size_t)m + 3);
    const int n = (int)(v->sites.size() / 3);

    // uniform bins with about two sites each, shaped like the domain
    double vol = dx * dy * dz;
    double h = std::cbrt(vol / std::max(1.0, n / 2.0));
    int gn[3] = {std::max(1, std::min(1024, (int)std::ceil(dx / h))), std::max(1, std::min(1024, (int)std::ceil(dy / h))),
                 std::max(1, std::min(1024, (int)std::ceil(dz / h)))};
    double gh[3] = {dx / gn[0], dy / gn[1], dz / gn[2]};
    size_t nbins = (size_t)gn[0] * gn[1] * gn[2];
    std::vector<int> boff(nbins + 1, 0), bin_of(n);
    for (int m = 0; m < n; m++) {
        const double* p = &v->sites[3 * (size_t)m];
        int b[3];
        for (int c = 0; c < 3; c++) b[c] = std::max(0, std::min(gn[c] - 1, (int)((p[c] - ext[c]) / gh[c])));
        bin_of[m] = (b[0] * gn[1] + b[1]) * gn[2] + b[2];
        boff[bin_of[m] + 1]++;
    }
    for (size_t b = 0; b < nbins; b++) boff[b + 1] += boff[b];
    std::vector<int> bid(n), fill(boff.begin(), boff.end() - 1);
    for (int m = 0; m < n; m++) bid[fill[bin_of[m]]++] = m;

    int rc = SKG_OK;
    std::string err;
    {
        cudaSetDevice(device);
        void* d[10] = {nullptr};
        size_t sz[10] = {3 * (size_t)n * 8, 6 * 8, (nbins + 1) * 4, (size_t)n * 4, (size_t)n * 4, (size_t)n * VMAXN * 4,
                         (size_t)n * 8, 3 * (size_t)n * 8, 6 * (size_t)n * 8, (size_t)n * 4};
        for (int q = 0; q < 10 && rc == SKG_OK; q++)
            if (cudaMalloc(&d[q], sz[q]) != cudaSuccess) { cudaGetLastError(); rc = SKG_ERR_OOM; err = "device allocation failed"; }
        if (rc == SKG_OK) {
            cudaMemcpy(d[0], v->sites.data(), sz[0], cudaMemcpyHostToDevice);
            cudaMemcpy(d[1], ext, sz[1], cudaMemcpyHostToDevice);
            cudaMemcpy(d[2], boff.data(), sz[2], cudaMemcpyHostToDevice);
            cudaMemcpy(d[3], bid.data(), sz[3], cudaMemcpyHostToDevice);
            BinGrid G;
            for (int c = 0; c < 3; c++) { G.lo[c] = ext[c]; G.h[c] = gh[c]; G.n[c] = gn[c]; }
            G.off = (const int*)d[2]; G.ids = (const int*)d[3];
            voronoi_cell_kernel<<<(n + 63) / 64, 64>>>((const double*)d[0], n, (const double*)d[1], G, (int*)d[4],
                                                       (int*)d[5], (double*)d[6], (double*)d[7], (double*)d[8], (int*)d[9]);
            cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) { rc = SKG_ERR_CUDA; err = cudaGetErrorString(e); }
        }
        if (rc == SKG_OK) {
            std::vector<int> cnt(n), ids((size_t)n * VMAXN), status(n);
            v->volume.resize(n); v->centroid.resize(3 * (size_t)n); v->bbox.resize(6 * (size_t)n);
            cudaMemcpy(cnt.data(), d[4], sz[4], cudaMemcpyDeviceToHost);
            cudaMemcpy(ids.data(), d[5], sz[5], cudaMemcpyDeviceToHost);
            cudaMemcpy(v->volume.data(), d[6], sz[6], cudaMemcpyDeviceToHost);
            cudaMemcpy(v->centroid.data(), d[7], sz[7], cudaMemcpyDeviceToHost);
            cudaMemcpy(v->bbox.data(), d[8], sz[8], cudaMemcpyDeviceToHost);
            cudaMemcpy(status.data(), d[9], sz[9], cudaMemcpyDeviceToHost);
            // cells beyond the device capacities (many neighbours, e.g. a sparse cell against a
            // dense region) are rebuilt on the host with larger ones
            BinGrid H;
            for (int c = 0; c < 3; c++) { H.lo[c] = ext[c]; H.h[c] = gh[c]; H.n[c] = gn[c]; }
            H.off = boff.data(); H.ids = bid.data();
            std::map<int, std::vector<int>> big;
            int bad = 0;
            for (int m = 0; m < n; m++) {
                if (!status[m]) continue;
                int hc = 0, hst = 0;
                std::vector<int> hid(HMAXN);
                double hv, hcen[3], hbb[6];
                voronoi_cell_t<HMAXP, HMAXT, HMAXC, HMAXN>(m, 0, v->sites.data(), ext, H, &hc, hid.data(), &hv, hcen,
                                                           hbb, &hst);
                if (hst) { bad++; continue; }
                hid.resize(hc);
                big[m] = hid;
                cnt[m] = hc;
                v->volume[m] = hv;
                std::copy(hcen, hcen + 3, &v->centroid[3 * (size_t)m]);
                std::copy(hbb, hbb + 6, &v->bbox[6 * (size_t)m]);
            }
            if (bad) { rc = SKG_ERR_INVALID; err = "Voronoi cell construction failed for " + std::to_string(bad) + " cells"; }
            v->noff.assign(n + 1, 0);
            for (int m = 0; m < n; m++) v->noff[m + 1] = v->noff[m] + cnt[m];
            v->nbr.resize(v->noff[n]);
            for (int m = 0; m < n; m++) {
                auto it = big.find(m);
                if (it != big.end()) std::copy(it->second.begin(), it->second.end(), &v->nbr[v->noff[m]]);
                else std::copy(&ids[(size_t)m * VMAXN], &ids[(size_t)m * VMAXN] + cnt[m], &v->nbr[v->noff[m]]);
            }
        }
        for (int q = 0; q < 10; q++) if (d[q]) cudaFree(d[q]);
    }
    if (rc != SKG_OK) { set_error(err); delete v; return rc; }

    // block lists: cells whose box (+-eps) overlaps each of nb^3 blocks (VoronoiMesh.cpp:334-390)
    int nb = std::max(3, std::min(1000, (int)(3. * std::pow(n, 1. / 3.))));
    v->nb = nb;
    size_t nb3 = (size_t)nb * nb * nb;
    std::vector<int64_t> bc(nb3 + 1, 0);
    auto cellindices = [&](const double* r, int* ijk) {   // Box::cellindices (Box.hpp:120-125)
        for (int c = 0; c < 3; c++) ijk[c] = std::max(0, std::min(nb - 1, (int)(nb * (r[c] - ext[c]) / (ext[c + 3] - ext[c]))));
    };
    for (int pass = 0; pass < 2; pass++) {
        std::vector<int64_t> pos;
        if (pass == 1) {
            for (size_t b = 0; b < nb3; b++) bc[b + 1] += bc[b];
            v->bids.resize(bc[nb3]);
            pos.assign(bc.begin(), bc.end() - 1);
        }
        for (int m = 0; m < n; m++) {
            double a[3], b[3];
            for (int c = 0; c < 3; c++) { a[c] = v->bbox[6 * (size_t)m + c] - eps; b[c] = v->bbox[6 * (size_t)m + 3 + c] + eps; }
            int i1[3], i2[3];
            cellindices(a, i1); cellindices(b, i2);
            for (int x = i1[0]; x <= i2[0]; x++)
                for (int y = i1[1]; y <= i2[1]; y++)
                    for (int z = i1[2]; z <= i2[2]; z++) {
                        size_t blk = ((size_t)x * nb + y) * nb + z;
                        if (pass == 0) bc[blk + 1]++;
                        else v->bids[pos[blk]++] = m;
                    }
        }
    }
    v->boff = bc;
    *out = v;
    return SKG_OK;
}

int skg_voronoi_sizes(const skg_voronoi* v, int32_t* nsites, int64_t* nnbr, int32_t* nb, int64_t* nblockids) {
    if (!v) return SKG_ERR_INVALID;
    if (nsites) *nsites = (int32_t)(v->sites.size() / 3);
    if (nnbr) *nnbr = (int64_t)v->nbr.size();
    if (nb) *nb = v->nb;
    if (nblockids) *nblockids = (int64_t)v->bids.size();
    return SKG_OK;
}

int skg_voronoi_arrays(const skg_voronoi* v, double* sites, int64_t* vnbr_offsets, int32_t* vnbr_ids, double* volume,
                       double* centroid, double* bbox, int64_t* block_offsets, int32_t* block_ids) {
    if (!v) return SKG_ERR_INVALID;
    if (sites) std::memcpy(sites, v->sites.data(), v->sites.size() * sizeof(double));
    if (vnbr_offsets) std::memcpy(vnbr_offsets, v->noff.data(), v->noff.size() * sizeof(int64_t));
    if (vnbr_ids) std::memcpy(vnbr_ids, v->nbr.data(), v->nbr.size() * sizeof(int32_t));
    if (volume) std::memcpy(volume, v->volume.data(), v->volume.size() * sizeof(double));
    if (centroid) std::memcpy(centroid, v->centroid.data(), v->centroid.size() * sizeof(double));
    if (bbox) std::memcpy(bbox, v->bbox.data(), v->bbox.size() * sizeof(double));
    if (block_offsets) std::memcpy(block_offsets, v->boff.data(), v->boff.size() * sizeof(int64_t));
    if (block_ids) std::memcpy(block_ids, v->bids.data(), v->bids.size() * sizeof(int32_t));
    return SKG_OK;
}

int skg_voronoi_grid(const skg_voronoi* v, skg_grid* g) {
    if (!v || !g) return SKG_ERR_INVALID;
    g->type = SKG_GRID_VORONOI;
    g->xmin = v->ext[0]; g->ymin = v->ext[1]; g->zmin = v->ext[2];
    g->xmax = v->ext[3]; g->ymax = v->ext[4]; g->zmax = v->ext[5];
    g->nsites = (int32_t)(v->sites.size() / 3);
    g->sites = v->sites.data();
    g->vnbr_offsets = v->noff.data();
    g->vnbr_ids = v->nbr.data();
    g->nb = v->nb;
    g->block_offsets = v->boff.data();
    g->block_ids = v->bids.data();
    g->cell_volume = v->volume.data();
    g->cell_bbox = v->bbox.data();
    return SKG_OK;
}

int skg_voronoi_destroy(skg_voronoi* v) { delete v; return SKG_OK; }

}  // extern "C"
