// skg_host.cpp -- host-side set-up of the library: tree topology and neighbour lists, the
// Sersic tables, the chunk parameters of the packet loop and the per-thread error message.
#include "skg_internal.h"
#include "skg_tree.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>

namespace skg {

static thread_local std::string g_error;
void set_error(const std::string& msg) { g_error = msg; }
const char* get_error() { return g_error.c_str(); }

// Sersic profile tables (SersicFunction.cpp:17-76): 101 logarithmic points s in [1e-6, 1e4],
// the deprojected density S(s) by trapezoid integration of the Abel integral in u, and the
// normalised cumulative mass M(s) by 33-point trapezoids between the points.
static double sersic_S(const double* sv, const double* Sv, double s) {
    if (s <= sv[0]) return Sv[0];
    if (s >= sv[100]) return Sv[100];
    int jl = -1, ju = 100;
    while (ju - jl > 1) { int jm = (ju + jl) >> 1; if (s < sv[jm]) ju = jm; else jl = jm; }
    int i = jl;
    double x = std::log10(s), x1 = std::log10(sv[i]), x2 = std::log10(sv[i + 1]);
    double f1 = Sv[i], f2 = Sv[i + 1];
    bool lg = f1 > 0 && f2 > 0;
    if (lg) { f1 = std::log10(f1); f2 = std::log10(f2); }
    double fx = f1 + ((x - x1) / (x2 - x1)) * (f2 - f1);
    return lg ? std::pow(10, fx) : fx;
}

void sersic_table(double n, double* sv, double* Sv, double* Mv) {
    const int Ns = 101;
    double b = 2.0 * n - 1.0 / 3.0 + 4.0 / 405.0 / n + 46.0 / 25515.0 / (n * n) + 131.0 / 1148175.0 / (n * n * n);
    double I0 = std::pow(b, 2.0 * n) / (M_PI * std::tgamma(2.0 * n + 1));
    const double logsmin = -6.0, dlogs = 10.0 / (Ns - 1.0);
    const int Nu = 10000;
    const double umax = std::sqrt(101.0 * 99.0), du = umax / Nu;
    for (int i = 0; i < Ns; i++) {
        double s = std::pow(10.0, logsmin + i * dlogs);
        sv[i] = s;
        double alpha = b * std::pow(s, 1.0 / n);
        double sum = 0.0;
        for (int j = 0; j <= Nu; j++) {
            double u = j * du, u2 = u * u;
            double w = (u > 1e-3) ? (std::pow(1.0 + u2, 2.0 * n) - 1.0) / u2
                                  : 2.0 * n + n * (2.0 * n - 1.0) * u2 + 2.0 / 3.0 * n * (2.0 * n - 1.0) * (n - 1.0) * u2 * u2;
            double term = 2.0 * std::exp(-alpha * (1.0 + u2)) / std::sqrt(w);
            sum += (j == 0 || j == Nu) ? 0.5 * term : term;
        }
        Sv[i] = I0 * std::pow(b, n) * std::pow(alpha, 1.0 - n) / M_PI * du * sum;
    }
    Mv[0] = 0.0;
    for (int i = 1; i < Ns; i++) {
        double ds = (sv[i] - sv[i - 1]) / 32.0, sum = 0.0;
        for (int j = 0; j <= 32; j++) {
            double s = sv[i - 1] + j * ds;
            double term = sersic_S(sv, Sv, s) * s * s * ds;
            sum += (j == 0 || j == 32) ? 0.5 * term : term;
        }
        Mv[i] = Mv[i - 1] + 4.0 * M_PI * sum;
    }
    for (int i = 0; i < Ns; i++) Mv[i] /= Mv[Ns - 1];
}

// MonteCarloSimulation::setChunkParams (MonteCarloSimulation.cpp:68-114), task-parallel mode:
// the packet count actually run per wavelength is totalChunks*chunksize >= packages.
void chunk_params(double packages, int Nthreads, int Nprocs, int Nlambda,
                  uint64_t& Nchunks, uint64_t& chunksize, uint64_t& Npp) {
    if (packages <= 0) { Nchunks = chunksize = Npp = 0; return; }
    if (Nthreads < 1) Nthreads = 1;
    if (Nprocs < 1) Nprocs = 1;
    int64_t totalChunks = (Nthreads == 1) ? 1
        : (int64_t)std::ceil(std::max(10. * double(Nthreads * Nprocs) / Nlambda, packages / 1e7));
    if (totalChunks % Nprocs) totalChunks = totalChunks + Nprocs - (totalChunks % Nprocs);
    chunksize = (uint64_t)std::ceil(packages / totalChunks);
    Nchunks = totalChunks / Nprocs;
    Npp = totalChunks * chunksize;
}

// ---------------------------------------------------------------------------------------------
// Tree topology.
//
// Nodes are created in breadth-first order (node 0 = root; the children of a node get
// consecutive ids), exactly as TreeDustGrid::setupSelfBefore visits and subdivides them
// (TreeDustGrid.cpp:80-98), so node ids, the leaf -> cell numbering (:106-116) and the
// octree index arithmetic of the Bookkeeping search agree with the reference.
//
// Neighbour lists follow the reference's incremental scheme because the ORDER of each list is
// observable (TreeNode::whichnode(wall, r) returns the first neighbour containing r): nodes are
// visited in id order, and each node hands its wall lists on to its children
// (OctTreeNode.cpp:67-180, BinTreeNode.cpp:75-320); finally each list is ordered by decreasing
// overlap area with std::sort (TreeNode.cpp:96-158).

static const int kOpposite[6] = {1, 0, 3, 2, 5, 4};   // BACK<->FRONT, LEFT<->RIGHT, BOTTOM<->TOP

void Tree::split(int l) {
    TNode& nd = nodes[l];
    int id0 = (int)nodes.size();
    double b[6]; std::memcpy(b, nd.box, sizeof(b));
    int lev = nd.level + 1;
    nodes[l].child = id0;
    if (type == SKG_GRID_OCTREE) {
        // OctTreeNode::createchildren_splitpoint at the centre (OctTreeNode.cpp:29-49)
        double cx = 0.5 * (b[0] + b[3]), cy = 0.5 * (b[1] + b[4]), cz = 0.5 * (b[2] + b[5]);
        const double xs[3] = {b[0], cx, b[3]}, ys[3] = {b[1], cy, b[4]}, zs[3] = {b[2], cz, b[5]};
        for (int o = 0; o < 8; o++) {
            int ix = o & 1, iy = (o >> 1) & 1, iz = (o >> 2) & 1;
            TNode c;
            c.box[0] = xs[ix]; c.box[1] = ys[iy]; c.box[2] = zs[iz];
            c.box[3] = xs[ix + 1]; c.box[4] = ys[iy + 1]; c.box[5] = zs[iz + 1];
            c.father = l; c.level = lev;
            nodes.push_back(c);
        }
    } else {
        // BinTreeNode::createchildren_splitdir with direction level % 3 (BinTreeNode.cpp:36-70)
        int d = nodes[l].level % 3;
        nodes[l].dir = (signed char)d;
        double c = 0.5 * (b[d] + b[d + 3]);
        TNode c0, c1;
        std::memcpy(c0.box, b, sizeof(b)); std::memcpy(c1.box, b, sizeof(b));
        c0.box[d + 3] = c; c1.box[d] = c;
        c0.father = c1.father = l; c0.level = c1.level = lev;
        nodes.push_back(c0); nodes.push_back(c1);
    }
}

static inline void erase_first(std::vector<int>& v, int x) {
    auto it = std::find(v.begin(), v.end(), x);
    if (it != v.end()) v.erase(it);
}

void Tree::make_neighbors(int wall1, int n1, int n2) {   // TreeNode::makeneighbors (TreeNode.cpp:183-188)
    nbrs[(size_t)n1 * 6 + wall1].push_back(n2);
    nbrs[(size_t)n2 * 6 + kOpposite[wall1]].push_back(n1);
}

// Hands the wall lists of node l on to its children.
void Tree::add_neighbors(int l) {
    const TNode& nd = nodes[l];
    if (nd.child < 0) return;
    int c = nd.child;
    auto lo = [&](int id, int ax) { return nodes[id].box[ax]; };
    auto hi = [&](int id, int ax) { return nodes[id].box[ax + 3]; };
    auto L = [&](int w) -> std::vector<int>& { return nbrs[(size_t)l * 6 + w]; };
    if (type == SKG_GRID_OCTREE) {
        // internal neighbours among the 8 children
        make_neighbors(1, c + 0, c + 1); make_neighbors(3, c + 0, c + 2); make_neighbors(5, c + 0, c + 4);
        make_neighbors(3, c + 1, c + 3); make_neighbors(5, c + 1, c + 5); make_neighbors(1, c + 2, c + 3);
        make_neighbors(5, c + 2, c + 6); make_neighbors(5, c + 3, c + 7); make_neighbors(1, c + 4, c + 5);
        make_neighbors(3, c + 4, c + 6); make_neighbors(3, c + 5, c + 7); make_neighbors(1, c + 6, c + 7);
        double xc = hi(c, 0), yc = hi(c, 1), zc = hi(c, 2);
        // for wall w of this node: the two axes spanning the wall, and the children on that side
        struct WallSpec { int a1, a2; int kids[4]; };
        static const WallSpec spec[6] = {
            {1, 2, {0, 2, 4, 6}},   // BACK   (x-): neighbours get the children at low x
            {1, 2, {1, 3, 5, 7}},   // FRONT  (x+)
            {0, 2, {0, 1, 4, 5}},   // LEFT   (y-)
            {0, 2, {2, 3, 6, 7}},   // RIGHT  (y+)
            {0, 1, {0, 1, 2, 3}},   // BOTTOM (z-)
            {0, 1, {4, 5, 6, 7}},   // TOP    (z+)
        };
        const double cen[3] = {xc, yc, zc};
        for (int w = 0; w < 6; w++) {
            std::vector<int> list = L(w);   // copy: make_neighbors may append to other lists
            const WallSpec& sp = spec[w];
            for (int nb : list) {
                erase_first(nbrs[(size_t)nb * 6 + kOpposite[w]], l);
                double c1 = cen[sp.a1], c2 = cen[sp.a2];
                bool lo1 = lo(nb, sp.a1) <= c1, hi1 = hi(nb, sp.a1) >= c1;
                bool lo2 = lo(nb, sp.a2) <= c2, hi2 = hi(nb, sp.a2) >= c2;
                // children order: (low a1, low a2), (high a1, low a2), (low a1, high a2), (high a1, high a2)
                if (lo1 && lo2) make_neighbors(kOpposite[w], nb, c + sp.kids[0]);
                if (hi1 && lo2) make_neighbors(kOpposite[w], nb, c + sp.kids[1]);
                if (lo1 && hi2) make_neighbors(kOpposite[w], nb, c + sp.kids[2]);
                if (hi1 && hi2) make_neighbors(kOpposite[w], nb, c + sp.kids[3]);
            }
        }
    } else {
        int d = nd.dir;
        double sc = hi(c, d);
        make_neighbors(2 * d + 1, c, c + 1);             // internal neighbour across the split
        for (int w = 0; w < 6; w++) {
            std::vector<int> list = L(w);
            int ax = w / 2;
            for (int nb : list) {
                erase_first(nbrs[(size_t)nb * 6 + kOpposite[w]], l);
                if (ax == d) {
                    // the wall perpendicular to the split touches one child only
                    make_neighbors(kOpposite[w], nb, (w % 2 == 0) ? c : c + 1);
                } else {
                    if (lo(nb, d) <= sc) make_neighbors(kOpposite[w], nb, c);
                    if (hi(nb, d) >= sc) make_neighbors(kOpposite[w], nb, c + 1);
                }
            }
        }
    }
    // the lists of a subdivided node are never consulted again
    for (int w = 0; w < 6; w++) { std::vector<int>().swap(L(w)); }
}

static double rect_overlap(double a1, double b1, double a2, double b2, double c1, double d1, double c2, double d2) {
    return std::max(std::min(a2, c2) - std::max(a1, c1), 0.) * std::max(std::min(b2, d2) - std::max(b1, d1), 0.);
}

void Tree::sort_neighbors(int l) {   // TreeNode::sortneighbors with the LargerOverlap ordering (TreeNode.cpp:96-158)
    const double* B = nodes[l].box;
    for (int w = 0; w < 6; w++) {
        int a1 = (w < 2) ? 1 : 0, a2 = (w < 4) ? 2 : 1;
        auto overlap = [&](int id) {
            const double* N = nodes[id].box;
            return rect_overlap(B[a1], B[a2], B[a1 + 3], B[a2 + 3], N[a1], N[a2], N[a1 + 3], N[a2 + 3]);
        };
        std::vector<int>& v = nbrs[(size_t)l * 6 + w];
        std::sort(v.begin(), v.end(), [&](int n1, int n2) { return overlap(n1) > overlap(n2); });
    }
}

void Tree::finish(bool with_neighbors) {
    ncells = 0;
    for (auto& nd : nodes) nd.cell = (nd.child < 0) ? ncells++ : -1;
    if (!with_neighbors) return;
    nbrs.assign(nodes.size() * 6, std::vector<int>());
    for (size_t l = 0; l < nodes.size(); l++) add_neighbors((int)l);
    for (size_t l = 0; l < nodes.size(); l++) if (nodes[l].child < 0) sort_neighbors((int)l);
}

void Tree::flatten() {
    size_t n = nodes.size();
    box.resize(6 * n); child.resize(n); father.resize(n); cell.resize(n); dir.resize(n);
    cell_node.assign(ncells, 0);
    nbroff.assign(6 * n + 1, 0);
    for (size_t l = 0; l < n; l++) {
        std::memcpy(&box[6 * l], nodes[l].box, 6 * sizeof(double));
        child[l] = nodes[l].child; father[l] = nodes[l].father; cell[l] = nodes[l].cell; dir[l] = nodes[l].dir;
        if (cell[l] >= 0) cell_node[cell[l]] = (int)l;
    }
    if (!nbrs.empty()) {
        for (size_t q = 0; q < 6 * n; q++) nbroff[q + 1] = nbroff[q] + (int64_t)nbrs[q].size();
        nbr.resize(nbroff[6 * n]);
        for (size_t q = 0; q < 6 * n; q++) std::copy(nbrs[q].begin(), nbrs[q].end(), nbr.begin() + nbroff[q]);
        std::vector<std::vector<int>>().swap(nbrs);
    }
}

void Tree::fill_grid(skg_grid* g) const {
    g->type = type;
    g->xmin = ext[0]; g->ymin = ext[1]; g->zmin = ext[2]; g->xmax = ext[3]; g->ymax = ext[4]; g->zmax = ext[5];
    g->nnodes = (int32_t)nodes.size();
    g->node_box = box.data(); g->node_child = child.data(); g->node_father = father.data();
    g->node_cell = cell.data(); g->node_dir = dir.data();
    g->nbr_offsets = nbr.empty() ? nullptr : nbroff.data();
    g->nbr_ids = nbr.empty() ? nullptr : nbr.data();
    g->search_method = SKG_SEARCH_NEIGHBOR;
}

// Level-synchronous subdivision by the criteria of TreeDustGrid::subdivide (TreeDustGrid.cpp:166-230):
// below or at minlevel always split; below maxlevel split when a stopping criterion fails
// (mass fraction, mean optical depth kappa_V M / V^(2/3), density dispersion); the per-node
// samples come from `sample` (a device kernel), one batch per level.
void Tree::build(int min_level, int max_level, double max_mass_fraction, double max_optical_depth,
                 double max_dens_disp, double total_mass,
                 const std::function<void(const std::vector<int>&, std::vector<double>&, std::vector<double>&,
                                          std::vector<double>&)>& sample) {
    nodes.clear();
    TNode root;
    std::memcpy(root.box, ext, sizeof(ext));
    root.father = -1; root.level = 0;
    nodes.push_back(root);
    size_t lev_begin = 0;
    const double kappaV = 2600.;   // Units::kappaV (Units.cpp:29)
    bool no_criteria = (max_optical_depth == 0 && max_mass_fraction == 0 && max_dens_disp == 0);
    while (lev_begin < nodes.size()) {
        size_t lev_end = nodes.size();
        int level = nodes[lev_begin].level;
        if (level >= max_level) break;
        std::vector<char> dosplit(lev_end - lev_begin, 0);
        if (level <= min_level || no_criteria) {
            std::fill(dosplit.begin(), dosplit.end(), 1);
        } else {
            std::vector<int> ids;
            for (size_t l = lev_begin; l < lev_end; l++) ids.push_back((int)l);
            std::vector<double> mass, rmin, rmax;
            sample(ids, mass, rmin, rmax);
            for (size_t q = 0; q < ids.size(); q++) {
                const double* b = nodes[ids[q]].box;
                double vol = (b[3] - b[0]) * (b[4] - b[1]) * (b[5] - b[2]);
                bool need = false;
                if (max_mass_fraction > 0 && mass[q] / total_mass >= max_mass_fraction) need = true;
                if (!need && max_optical_depth > 0 && kappaV * mass[q] / std::pow(vol, 2. / 3.) >= max_optical_depth) need = true;
                if (!need && max_dens_disp > 0) {
                    double dd = rmax[q] > 0 ? (rmax[q] - rmin[q]) / rmax[q] : 0;
                    if (dd >= max_dens_disp) need = true;
                }
                dosplit[q] = need;
            }
        }
        for (size_t l = lev_begin; l < lev_end; l++) if (dosplit[l - lev_begin]) split((int)l);
        lev_begin = lev_end;
    }
}

// ---------------------------------------------------------------------------------------------
// Lattice form of the rope tree (layout in skg_tree.h).  Every node box must be an interval of the
// root's extent halved l_a times along each axis a (l_a <= 20); the codes are checked against the
// FP64 boxes to 1e-6 of the node width.  Leaves are re-ordered by cell number, so that a leaf
// reference is the cell number and the record carries no separate cell field; leaf references in
// the ropes and internal records are translated accordingly.  Leaves the form unchanged (64-byte
// records) when a box does not fit or the references do not fit 25 bits.
static void build_lattice_records(const skg_grid& g, const std::vector<int>& order, const std::vector<int>& ref,
                                  int nleaf, int nint, RopeTree& out) {
    const int n = g.nnodes;
    const double org[3] = {g.xmin, g.ymin, g.zmin};
    const double wid[3] = {g.xmax - g.xmin, g.ymax - g.ymin, g.zmax - g.zmin};
    if (nleaf >= (1 << 25) || nint >= (1 << 25) - 1) return;
    std::vector<uint32_t> code(3 * (size_t)n);
    for (int l = 0; l < n; l++) {
        const double* b = g.node_box + 6 * (size_t)l;
        for (int a = 0; a < 3; a++) {
            const double w = b[a + 3] - b[a];
            if (!(w > 0) || !(wid[a] > 0)) return;
            const int lev = (int)std::lround(std::log2(wid[a] / w));
            if (lev < 0 || lev > 20) return;
            const double unit = std::ldexp(wid[a], -lev);
            const long long i = std::llround((b[a] - org[a]) / unit);
            if (i < 0 || i >= (1ll << lev)) return;
            const double tol = 1e-6 * unit;
            if (std::fabs(b[a] - (org[a] + (double)i * unit)) > tol ||
                std::fabs(b[a + 3] - (org[a] + (double)(i + 1) * unit)) > tol) return;
            code[3 * (size_t)l + a] = (uint32_t)((2 * i + 1) << (20 - lev));
        }
    }
    std::vector<int> leaf_cell(nleaf, -1);
    std::vector<char> seen(nleaf, 0);
    for (int l = 0; l < n; l++) {
        if (g.node_child[l] >= 0) continue;
        const int c = g.node_cell[l];
        if (c < 0 || c >= nleaf || seen[c]) return;      // cells must number the leaves 0..nleaf-1
        seen[c] = 1;
        leaf_cell[ref[l]] = c;
    }
    auto cref = [&](int r) { return r >= 0 ? leaf_cell[r] : r; };
    auto as_i = [](float f) { int v; std::memcpy(&v, &f, 4); return v; };
    auto as_f = [](int v) { float f; std::memcpy(&f, &v, 4); return f; };
    for (int a = 0; a < 3; a++) {
        out.lorg[a] = (float)org[a];
        out.lunit[a] = std::ldexp((float)wid[a], -21);
    }
    out.prec.assign(2 * (size_t)nleaf, uint4{0, 0, 0, 0});
    for (int l : order) {
        const uint32_t* c = code.data() + 3 * (size_t)l;
        if (g.node_child[l] >= 0) {
            const int j = -ref[l] - 2;
            float4& h = out.irec[3 * (size_t)j];
            // the split point is the node's centre, as the walls of its children compute it
            h.x = std::fmaf((float)c[0], out.lunit[0], out.lorg[0]);
            h.y = std::fmaf((float)c[1], out.lunit[1], out.lorg[1]);
            h.z = std::fmaf((float)c[2], out.lunit[2], out.lorg[2]);
            for (int q = 1; q <= 2; q++) {
                float4& v = out.irec[3 * (size_t)j + q];
                v = float4{as_f(cref(as_i(v.x))), as_f(cref(as_i(v.y))), as_f(cref(as_i(v.z))), as_f(cref(as_i(v.w)))};
            }
            continue;
        }
        const int li = ref[l], cell = leaf_cell[li];
        const float4 r03 = out.lrec[4 * (size_t)li + 2], r45 = out.lrec[4 * (size_t)li + 3];
        const int rope[6] = {as_i(r03.x), as_i(r03.y), as_i(r03.z), as_i(r03.w), as_i(r45.x), as_i(r45.y)};
        uint32_t bits[5] = {0, 0, 0, 0, 0};
        for (int w = 0; w < 6; w++) {
            const int r = rope[w];
            const uint64_t v = (r == -1) ? 0x3FFFFFFull : (r >= 0) ? (uint64_t)leaf_cell[r] : (uint64_t)((1 << 25) + (-r - 2));
            const int bit = 26 * w, wd = bit >> 5, sh = bit & 31;
            const uint64_t x = v << sh;
            bits[wd] |= (uint32_t)x;
            if (wd + 1 < 5) bits[wd + 1] |= (uint32_t)(x >> 32);
        }
        const uint64_t box = (uint64_t)c[0] | ((uint64_t)c[1] << 21) | ((uint64_t)c[2] << 42);
        out.prec[2 * (size_t)cell] = uint4{0u, (uint32_t)box, (uint32_t)(box >> 32), bits[0]};
        out.prec[2 * (size_t)cell + 1] = uint4{bits[1], bits[2], bits[3], bits[4]};
    }
    out.root_ref = cref(out.root_ref);
    out.lattice = true;
    std::vector<float4>().swap(out.lrec);
    for (int m = 0; m < nleaf; m++) out.cell_leaf[m] = m;
}

// ---------------------------------------------------------------------------------------------
// Rope-linked tree for the FP32 walk.
//
// Leaves are numbered in depth-first order (children in order: for an octree the Morton order of
// the leaves), so that leaves met in sequence along a ray sit close together in memory.  Each
// leaf face carries a rope: the deepest node beyond the face whose box covers the whole face
// (Havran's neighbour links).  A step then follows the rope of the exit wall -- to the next leaf
// directly, or to a node from which the point descends one or two levels.
void build_rope_tree(const skg_grid& g, RopeTree& out, bool allow_lattice) {
    const int n = g.nnodes;
    std::vector<int> ref(n, -1);
    std::vector<int> order;            // depth-first visit order
    order.reserve(n);
    std::vector<int> stack{0};
    int nleaf = 0, nint = 0;
    while (!stack.empty()) {
        int l = stack.back(); stack.pop_back();
        order.push_back(l);
        int c0 = g.node_child[l];
        if (c0 < 0) { ref[l] = nleaf++; continue; }
        ref[l] = -(nint++ + 2);
        int nch = (g.node_dir[l] < 0) ? 8 : 2;
        for (int c = nch - 1; c >= 0; c--) stack.push_back(c0 + c);
    }
    out.root_ref = ref[0];
    out.lrec.assign(4 * (size_t)nleaf, float4{0, 0, 0, 0});
    out.irec.assign(3 * (size_t)nint, float4{0, 0, 0, 0});
    int ncells = 0;
    for (int l = 0; l < n; l++) if (g.node_cell[l] >= 0) ncells = std::max(ncells, g.node_cell[l] + 1);
    out.cell_leaf.assign(ncells, -1);
    const double ext[6] = {g.xmin, g.ymin, g.zmin, g.xmax, g.ymax, g.zmax};
    auto box = [&](int l) { return g.node_box + 6 * (size_t)l; };
    auto as_f = [](int v) { float f; std::memcpy(&f, &v, 4); return f; };

    for (int l : order) {
        const double* b = box(l);
        int c0 = g.node_child[l];
        if (c0 >= 0) {
            int j = -ref[l] - 2;
            const double* s = box(c0);           // the split point is child 0's upper corner
            int d = g.node_dir[l];
            int nch = (d < 0) ? 8 : 2;
            int ch[8];
            for (int c = 0; c < 8; c++) ch[c] = (c < nch) ? ref[c0 + c] : -1;
            out.irec[3 * (size_t)j] = float4{(float)s[3], (float)s[4], (float)s[5], as_f(d)};
            out.irec[3 * (size_t)j + 1] = float4{as_f(ch[0]), as_f(ch[1]), as_f(ch[2]), as_f(ch[3])};
            out.irec[3 * (size_t)j + 2] = float4{as_f(ch[4]), as_f(ch[5]), as_f(ch[6]), as_f(ch[7])};
            continue;
        }
        int li = ref[l];
        int rope[6];
        for (int w = 0; w < 6; w++) {
            int a = w / 2;
            bool up = (w % 2) == 1;
            double c = up ? b[a + 3] : b[a];
            if ((up && c >= ext[a + 3]) || (!up && c <= ext[a])) { rope[w] = -1; continue; }
            // descend from the root while one child covers the whole face region
            int node = 0;
            while (g.node_child[node] >= 0) {
                int k0 = g.node_child[node];
                const double* sp = box(k0);
                int d = g.node_dir[node];
                int sel = 0;
                bool split_face = false;
                for (int ax = 0; ax < 3 && !split_face; ax++) {
                    if (d >= 0 && ax != d) continue;
                    double s = sp[ax + 3];
                    bool upper;
                    if (ax == a) upper = up ? (c >= s) : (c > s);   // the slab just beyond the face
                    else if (b[ax + 3] <= s) upper = false;
                    else if (b[ax] >= s) upper = true;
                    else { split_face = true; break; }
                    if (upper) sel |= (d < 0) ? (1 << ax) : 1;
                }
                if (split_face) break;
                node = k0 + sel;
            }
            rope[w] = ref[node];
        }
        int cell = g.node_cell[l];
        out.cell_leaf[cell] = li;
        out.lrec[4 * (size_t)li] = float4{(float)b[0], (float)b[1], (float)b[2], 0.f};
        out.lrec[4 * (size_t)li + 1] = float4{(float)b[3], (float)b[4], (float)b[5], as_f(cell)};
        out.lrec[4 * (size_t)li + 2] = float4{as_f(rope[0]), as_f(rope[1]), as_f(rope[2]), as_f(rope[3])};
        out.lrec[4 * (size_t)li + 3] = float4{as_f(rope[4]), as_f(rope[5]), 0.f, 0.f};
    }
    if (allow_lattice) build_lattice_records(g, order, ref, nleaf, nint, out);
}

// Builds the topology from explicit decisions (split[l] for node l in creation order).
void Tree::build_from_splits(const uint8_t* splitv, int64_t nsplit) {
    nodes.clear();
    TNode root;
    std::memcpy(root.box, ext, sizeof(ext));
    root.father = -1; root.level = 0;
    nodes.push_back(root);
    for (size_t l = 0; l < nodes.size(); l++)
        if ((int64_t)l < nsplit && splitv[l]) split((int)l);
}

}  // namespace skg
