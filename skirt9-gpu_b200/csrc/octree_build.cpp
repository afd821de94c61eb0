// Host-side octree construction for standalone scenes (in the drop-in case SKIRT builds its own
// tree and hands the flattened arrays to skgpu_upload_grid_octree).
//
// Construction follows the reference's policy and data structure so that the exported arrays have
// the same form as TreeSpatialGrid's:
//  - DensityTreePolicy::constructTree / needsSubdivide (SKIRT/core/DensityTreePolicy.cpp:88-245):
//    level by level; a node is subdivided below minLevel, never at maxLevel, and otherwise when the
//    dust mass fraction estimated from random density samples (mean density x volume) exceeds
//    maxDustFraction;
//  - OctTreeNode::createChildren (OctTreeNode.cpp:15-25): 8 children with consecutive ids in
//    x-fastest order;
//  - TreeNode/OctTreeNode neighbour bookkeeping (TreeNode.cpp:87-130, OctTreeNode.cpp:46-138):
//    siblings become neighbours, the parent's neighbours on each wall are replaced by the children
//    they touch; at the end each wall's list is sorted by decreasing overlap area
//    (TreeNode::sortNeighbors, TreeNode.cpp:200-209).
// The cell densities are the mean geometry density over random sample points per leaf
// (the reference's PropertySampler with numDensitySamples, MediumSystem.cpp:100-160).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/skgpu.h"

namespace {

struct Node
{
    double b[6];  // xmin, ymin, zmin, xmax, ymax, zmax
    int level;
    int firstChild = -1;
    std::vector<int> nb[6];  // BACK, FRONT, LEFT, RIGHT, BOTTOM, TOP
};

enum { BACK = 0, FRONT, LEFT, RIGHT, BOTTOM, TOP };

// splitmix64 stream for the sample positions
struct Rng
{
    uint64_t s;
    double uniform()
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    }
};

// normalised geometry densities (unit total mass)
struct Geometry
{
    int kind;
    double p[6];
    double rho0;

    void setup()
    {
        if (kind == SKGPU_GEOM_EXPDISK)
        {
            // ExpDiskGeometry::setupSelfBefore (ExpDiskGeometry.cpp:13-27)
            double hR = p[0], hz = p[1], Rmin = p[2], Rmax = p[3], zmax = p[4];
            double intphi = 2.0 * M_PI;
            double intz = (zmax > 0) ? -2.0 * hz * std::expm1(-zmax / hz) : 2.0 * hz;
            double tmin = (Rmin > 0) ? std::exp(-Rmin / hR) * (1.0 + Rmin / hR) : 1.0;
            double tmax = (Rmax > 0) ? std::exp(-Rmax / hR) * (1.0 + Rmax / hR) : 0.0;
            double intR = hR * hR * (tmin - tmax);
            rho0 = 1.0 / (intR * intphi * intz);
        }
        else
        {
            // ShellGeometry: rho = A r^-p between rmin and rmax, unit mass
            double rmin = p[0], rmax = p[1], e = p[2];
            double integral = std::fabs(3.0 - e) < 1e-12 ? std::log(rmax / rmin)
                                                          : (std::pow(rmax, 3.0 - e) - std::pow(rmin, 3.0 - e)) / (3.0 - e);
            rho0 = 1.0 / (4.0 * M_PI * integral);
        }
    }

    double density(double x, double y, double z) const
    {
        if (kind == SKGPU_GEOM_EXPDISK)
        {
            double R = std::sqrt(x * x + y * y), az = std::fabs(z);
            if (p[3] > 0 && R > p[3]) return 0.;
            if (p[4] > 0 && az > p[4]) return 0.;
            if (R < p[2]) return 0.;
            return rho0 * std::exp(-R / p[0]) * std::exp(-az / p[1]);
        }
        double r = std::sqrt(x * x + y * y + z * z);
        if (r < p[0] || r > p[1]) return 0.;
        return rho0 * std::pow(r, -p[2]);
    }
};

double meanDensity(const Geometry& g, const double* b, int n, Rng& rng)
{
    double sum = 0.;
    for (int i = 0; i < n; ++i)
    {
        double x = b[0] + rng.uniform() * (b[3] - b[0]);
        double y = b[1] + rng.uniform() * (b[4] - b[1]);
        double z = b[2] + rng.uniform() * (b[5] - b[2]);
        sum += g.density(x, y, z);
    }
    return sum / n;
}

double volume(const double* b) { return (b[3] - b[0]) * (b[4] - b[1]) * (b[5] - b[2]); }

void makeNeighbors(std::vector<Node>& v, int wall, int a, int b)
{
    static const int complement[6] = {FRONT, BACK, RIGHT, LEFT, TOP, BOTTOM};
    v[a].nb[wall].push_back(b);
    v[b].nb[complement[wall]].push_back(a);
}

void deleteNeighbor(std::vector<Node>& v, int node, int wall, int which)
{
    auto& l = v[node].nb[wall];
    auto it = std::find(l.begin(), l.end(), which);
    if (it != l.end()) l.erase(it);
}

void subdivide(std::vector<Node>& v, int id)
{
    int c = static_cast<int>(v.size());
    v[id].firstChild = c;
    double x0 = v[id].b[0], y0 = v[id].b[1], z0 = v[id].b[2], x1 = v[id].b[3], y1 = v[id].b[4], z1 = v[id].b[5];
    double xc = 0.5 * (x0 + x1), yc = 0.5 * (y0 + y1), zc = 0.5 * (z0 + z1);
    for (int k = 0; k < 8; ++k)
    {
        Node n;
        n.level = v[id].level + 1;
        n.b[0] = (k & 1) ? xc : x0;
        n.b[3] = (k & 1) ? x1 : xc;
        n.b[1] = (k & 2) ? yc : y0;
        n.b[4] = (k & 2) ? y1 : yc;
        n.b[2] = (k & 4) ? zc : z0;
        n.b[5] = (k & 4) ? z1 : zc;
        v.push_back(n);
    }
    // siblings
    const int pairs[12][3] = {{FRONT, 0, 1}, {RIGHT, 0, 2}, {TOP, 0, 4}, {RIGHT, 1, 3}, {TOP, 1, 5}, {FRONT, 2, 3},
                              {TOP, 2, 6},   {TOP, 3, 7},   {FRONT, 4, 5}, {RIGHT, 4, 6}, {RIGHT, 5, 7}, {FRONT, 6, 7}};
    for (const auto& q : pairs) makeNeighbors(v, q[0], c + q[1], c + q[2]);
    // the parent's neighbours on each wall now border the children they touch
    struct WallSpec { int wall, back, a0, a1; int kids[4]; };
    // for each wall: the complementary wall on the neighbour, the two transverse axes, the 4 children on the wall
    const WallSpec specs[6] = {{BACK, FRONT, 1, 2, {0, 2, 4, 6}},  {FRONT, BACK, 1, 2, {1, 3, 5, 7}},
                               {LEFT, RIGHT, 0, 2, {0, 1, 4, 5}},  {RIGHT, LEFT, 0, 2, {2, 3, 6, 7}},
                               {BOTTOM, TOP, 0, 1, {0, 1, 2, 3}},  {TOP, BOTTOM, 0, 1, {4, 5, 6, 7}}};
    double ctr[3] = {xc, yc, zc};
    for (const auto& sp : specs)
    {
        std::vector<int> list = v[id].nb[sp.wall];
        for (int nbId : list)
        {
            deleteNeighbor(v, nbId, sp.back, id);
            const double* nb = v[nbId].b;
            double c0 = ctr[sp.a0], c1 = ctr[sp.a1];
            bool lo0 = nb[sp.a0] <= c0, hi0 = nb[3 + sp.a0] >= c0;
            bool lo1 = nb[sp.a1] <= c1, hi1 = nb[3 + sp.a1] >= c1;
            // children on the wall in order (low,low), (high,low), (low,high), (high,high) of the two axes
            if (lo0 && lo1) makeNeighbors(v, sp.back, nbId, c + sp.kids[0]);
            if (hi0 && lo1) makeNeighbors(v, sp.back, nbId, c + sp.kids[1]);
            if (lo0 && hi1) makeNeighbors(v, sp.back, nbId, c + sp.kids[2]);
            if (hi0 && hi1) makeNeighbors(v, sp.back, nbId, c + sp.kids[3]);
        }
    }
}

double overlap(const double* a, const double* b, int wall)
{
    int u = (wall < 2) ? 1 : 0, w = (wall < 4) ? 2 : 1;
    double du = std::max(std::min(a[3 + u], b[3 + u]) - std::max(a[u], b[u]), 0.);
    double dw = std::max(std::min(a[3 + w], b[3 + w]) - std::max(a[w], b[w]), 0.);
    return du * dw;
}

}  // namespace

struct skgpu_octree
{
    std::vector<Node> nodes;
    std::vector<int> cellOfNode;
    std::vector<double> cellDensity;
    int numCells = 0;
    size_t numNb = 0;
};

extern "C" {

int skgpu_octree_build(const skgpu_octree_spec* spec, skgpu_octree** out)
{
    if (!spec || !out) return SKGPU_ERR_ARG;
    *out = nullptr;
    if (spec->geometry != SKGPU_GEOM_EXPDISK && spec->geometry != SKGPU_GEOM_SHELL) return SKGPU_ERR_ARG;
    if (spec->max_level < 0 || spec->max_level > 20 || spec->min_level < 0 || spec->num_subdivision_samples < 1
        || spec->num_density_samples < 1)
        return SKGPU_ERR_ARG;
    Geometry g;
    g.kind = spec->geometry;
    std::memcpy(g.p, spec->params, sizeof g.p);
    g.setup();
    auto* t = new skgpu_octree();
    Node root;
    std::memcpy(root.b, spec->extent, sizeof root.b);
    root.level = 0;
    t->nodes.push_back(root);
    Rng rng{spec->seed};
    size_t lbeg = 0, lend = 1;
    while (lend != lbeg)
    {
        std::vector<char> divide(lend - lbeg, 0);
        for (size_t l = lbeg; l < lend; ++l)
        {
            const Node& n = t->nodes[l];
            bool d;
            if (n.level < spec->min_level)
                d = true;
            else if (n.level >= spec->max_level)
                d = false;
            else
                d = meanDensity(g, n.b, spec->num_subdivision_samples, rng) * volume(n.b) > spec->max_dust_fraction;
            divide[l - lbeg] = d;
        }
        for (size_t l = lbeg; l < lend; ++l)
            if (divide[l - lbeg]) subdivide(t->nodes, static_cast<int>(l));
        lbeg = lend;
        lend = t->nodes.size();
    }
    // sort each wall's neighbours by decreasing overlap area
    for (Node& n : t->nodes)
        for (int wall = 0; wall < 6; ++wall)
        {
            const double* base = n.b;
            std::sort(n.nb[wall].begin(), n.nb[wall].end(), [&](int a, int b) {
                return overlap(base, t->nodes[a].b, wall) > overlap(base, t->nodes[b].b, wall);
            });
            t->numNb += n.nb[wall].size();
        }
    // leaves numbered depth-first, children in OctTreeNode order (x fastest): the cells follow a
    // Morton curve, so the walker's per-cell records of cells close in space lie close in memory
    // (TreeSpatialGrid numbers them level by level; only the numbering differs)
    t->cellOfNode.assign(t->nodes.size(), -1);
    {
        std::vector<int> stack{0};
        while (!stack.empty())
        {
            int l = stack.back();
            stack.pop_back();
            const Node& n = t->nodes[l];
            if (n.firstChild < 0)
            {
                t->cellOfNode[l] = t->numCells++;
                continue;
            }
            for (int q = 7; q >= 0; --q) stack.push_back(n.firstChild + q);
        }
    }
    t->cellDensity.resize(t->numCells);
    for (size_t l = 0; l < t->nodes.size(); ++l)
        if (t->cellOfNode[l] >= 0)
            t->cellDensity[t->cellOfNode[l]] = meanDensity(g, t->nodes[l].b, spec->num_density_samples, rng);
    *out = t;
    return SKGPU_OK;
}

int skgpu_octree_sizes(const skgpu_octree* t, int32_t* num_nodes, int32_t* num_cells, int64_t* num_nb)
{
    if (!t || !num_nodes || !num_cells || !num_nb) return SKGPU_ERR_ARG;
    *num_nodes = static_cast<int32_t>(t->nodes.size());
    *num_cells = t->numCells;
    *num_nb = static_cast<int64_t>(t->numNb);
    return SKGPU_OK;
}

int skgpu_octree_export(const skgpu_octree* t, double* bounds, int32_t* cell_index, int32_t* child_begin,
                        int32_t* child_count, int32_t* child_index, int32_t* nb_begin, int32_t* nb_index,
                        double* cell_density)
{
    if (!t) return SKGPU_ERR_ARG;
    size_t nn = t->nodes.size();
    int32_t childPos = 0;
    int64_t nbPos = 0;
    for (size_t l = 0; l < nn; ++l)
    {
        const Node& n = t->nodes[l];
        if (bounds) std::memcpy(bounds + 6 * l, n.b, sizeof n.b);
        if (cell_index) cell_index[l] = t->cellOfNode[l];
        if (child_begin) child_begin[l] = childPos;
        if (child_count) child_count[l] = n.firstChild >= 0 ? 8 : 0;
        if (n.firstChild >= 0)
        {
            if (child_index)
                for (int k = 0; k < 8; ++k) child_index[childPos + k] = n.firstChild + k;
            childPos += 8;
        }
        for (int wall = 0; wall < 6; ++wall)
        {
            if (nb_begin) nb_begin[6 * l + wall] = static_cast<int32_t>(nbPos);
            for (int id : n.nb[wall])
            {
                if (nb_index) nb_index[nbPos] = id;
                nbPos++;
            }
        }
    }
    if (nb_begin) nb_begin[6 * nn] = static_cast<int32_t>(nbPos);
    if (cell_density) std::copy(t->cellDensity.begin(), t->cellDensity.end(), cell_density);
    return SKGPU_OK;
}

void skgpu_octree_free(skgpu_octree* t) { delete t; }

}  // extern "C"
