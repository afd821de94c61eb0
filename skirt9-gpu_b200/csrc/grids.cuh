// Spatial-grid walkers of the tracer. Each walker is a device-side path segment generator with
// the interface of SKIRT's PathSegmentGenerator (start / next / m / ds). The *Exact walkers keep
// the reference generators' FP64 operation order with separate roundings, so that for identical
// rays they return the same cell sequences and segment lengths as the CPU code:
//   CartesianExact  <- CartesianSpatialGrid::MySegmentGenerator::next   (CartesianSpatialGrid.cpp:77-155)
//   OctreeExact     <- TreeSpatialGrid::MySegmentGenerator::next        (TreeSpatialGrid.cpp:143-228)
//   AdaptiveMeshExact <- AdaptiveMeshSnapshot::MySegmentGenerator::next (AdaptiveMeshSnapshot.cpp:378-449)
//   VoronoiExact    <- VoronoiMeshSnapshot::MySegmentGenerator::next    (VoronoiMeshSnapshot.cpp:1089-1222)
//   TetraExact      <- TetraMeshSpatialGrid::MySegmentGenerator::next   (TetraMeshSpatialGrid.cpp:688-831)
// and PathSegmentGenerator::moveInside (SKIRT/utils/PathSegmentGenerator.cpp:11-112).
#pragma once

#include "common.cuh"

namespace skg {

enum GenState { GS_UNKNOWN = 0, GS_INSIDE = 1, GS_OUTSIDE = 2 };

// All device-resident grid data. Only the members of the uploaded grid kind are set.
struct GridDev
{
    int kind;
    double ext[6];  // xmin, ymin, zmin, xmax, ymax, zmax
    double eps;
    int numCells;

    // Cartesian: borders (nx+1, ny+1, nz+1 entries)
    const double* xb;
    const double* yb;
    const double* zb;
    int nx, ny, nz;

    // octree: per node bounds (6 doubles), cell index (-1 non-leaf), first child (-1 leaf),
    // neighbour CSR per (node, wall)
    const double* tBounds;
    const int* tCell;
    const int* tChild;
    const int* tNbBegin;
    const int* tNb;
    int tNodes;
    // adaptive mesh (shares tBounds, tCell, tNbBegin, tNb with the octree, one neighbour per leaf
    // wall): per node the subdivision nx, ny, nz (0 for leaves) and the first entry of its
    // children in amChild (local Morton order, x fastest)
    const int* amDiv;
    const int* amChildBegin;
    const int* amChild;
    // leaf-indexed 64-byte records of the production walker (four int4 per cell):
    //   [0] wall indices x lo|hi<<16, y, z (16 bits each, into the lattice wall tables), FP32 density
    //   [1] neighbour-list base, 9-bit cumulative wall offsets (64 bits), leaf node id
    //   [2] [3] per wall the single positive-overlap neighbour (-1: domain wall, -2: scan the list)
    // and the positive-overlap neighbour lists (overlap-sorted, cell indices) of every leaf wall
    const int4* tRec;
    const int* tLeafNb;
    // the octree's lattice: every wall coordinate of a tree of depth L <= 15 built by halving is one
    // of 2^L + 1 FP64 values per axis (a child's bounds are copies of its parent's bounds and centre)
    const double* tWall;   // 3 x tWallN wall coordinates (x, y, z)
    int tWallN;            // 2^L + 1, or 0 when the tree is not such a lattice (no production records)

    // Voronoi: sites, neighbour CSR (negative = wall), uniform site-search grid
    const double* vSites;
    const int* vNbBegin;
    const int* vNb;
    int vN;
    const float4* vRec;    // FP32 walker: one record per cell (site, faces, neighbour record offsets)
    const int* vRecOff;    // record offset of each cell (16-byte units)
    int vGridN;            // blocks per dimension of the site search grid
    const int* vBlkBegin;  // vGridN^3 + 1
    const int* vBlkSites;  // site indices per block
    const int* vBlkRep;    // vGridN^3: a site in or near each block (start of the greedy locate)
    const double* vBox;    // per cell its enclosing box (secondary launch), or null

    // tetra: vertices, vertex indices (4 per tet), face normals (12 per tet), neighbour tet and
    // face per face, tet bounding boxes, uniform tet-search grid
    const double* teVerts;
    const int* teTet;
    const double* teNormals;
    const int* teNTet;
    const int* teNFace;
    const double* teBox;
    int teN;
    int teGridN;
    const int* teBlkBegin;
    const int* teBlkTets;
    const struct TetRec* teRec;  // FP32 walker: one cache-line record per tetrahedron
    // 1D spherical: sNr radial cells between the sNr + 1 ascending border radii sRv
    const double* sRv;
    int sNr;
    // 2D cylindrical: cNR radial x cNz vertical cells between the borders cRv and czv
    const double* cRv;
    const double* czv;
    int cNR, cNz;
    // 2D spherical: s2Nr radial x s2Nt polar cells; radial borders, polar borders and their cosines
    const double* s2r;
    const double* s2t;
    const double* s2c;
    int s2Nr, s2Nt;
    // 3D spherical: radial, polar (+ cosines) and azimuthal (+ sines, cosines) borders, path step
    const double* s3r;
    const double* s3t;
    const double* s3c;
    const double* s3p;
    const double* s3s;
    const double* s3k;
    int s3Nr, s3Nt, s3Np;
    double s3eps;
    // 3D cylindrical: radial, azimuthal (+ sines, cosines) and vertical borders, path step, real hole
    const double* c3r;
    const double* c3p;
    const double* c3s;
    const double* c3k;
    const double* c3z;
    int c3Nr, c3Np, c3Nz, c3Hole;
    double c3eps;
    const int* teBlkRep;         // teGridN^3: a tetrahedron overlapping each block (start of the walking locate)
};

// Per-tetrahedron record of the production walker, one 128-byte cache line: the four face planes
// n_f . x = c_f (outward FP32 unit normal, FP64 offset in global coordinates) and the neighbour
// across each face with the face index on its side. The two tetrahedra sharing a face hold exactly
// negated copies of one plane, so a point is never inside both (or neither) of them.
struct alignas(128) TetRec
{
    double c[4];
    float n[12];
    int nb[4];    // neighbour across face f, -1 on the hull
    int nface;    // neighbour's face index for face f in bits 8f..8f+7
    int pad[7];
};
static_assert(sizeof(TetRec) == 128, "one cache line per tetrahedron");

// ---------------------------------------------------------------------------------------------
// common generator state (PathSegmentGenerator)
// ---------------------------------------------------------------------------------------------
struct GenBase
{
    using Acc = double;  // accumulator type of optical depth and path length along the walk
    // the wavefront runs peel-off and propagation rays as two concurrent traversal kernels
    static constexpr bool kSplit = true;
    double rx, ry, rz, kx, ky, kz;
    double ds;
    int m;
    int state;

    SKG_D void startRay(double x, double y, double z, double ux, double uy, double uz)
    {
        state = GS_UNKNOWN;
        rx = x; ry = y; rz = z;
        kx = ux; ky = uy; kz = uz;
        m = -1;
        ds = 0.;
    }
    // number density of the cell of the segment just returned
    SKG_D double density(const double* dens) const { return dens[m]; }

    SKG_D void propagater(double d)
    {
        rx = xadd(rx, xmul(kx, d));
        ry = xadd(ry, xmul(ky, d));
        rz = xadd(rz, xmul(kz, d));
    }
    SKG_D static bool boxContains(const double* b, double x, double y, double z)
    {
        return x >= b[0] && x <= b[3] && y >= b[1] && y <= b[4] && z >= b[2] && z <= b[5];
    }
    // PathSegmentGenerator::moveInside (PathSegmentGenerator.cpp:11-112)
    SKG_D bool moveInside(const double* b, double eps)
    {
        m = -1;
        ds = 0.;
        state = GS_OUTSIDE;
        double cumds = 0.;
        if (rx <= b[0])
        {
            if (kx <= 0.0) return false;
            double d = (b[0] - rx) / kx;
            rx = xadd(b[0], eps);
            ry = xadd(ry, xmul(ky, d));
            rz = xadd(rz, xmul(kz, d));
            cumds = xadd(cumds, d);
        }
        else if (rx >= b[3])
        {
            if (kx >= 0.0) return false;
            double d = (b[3] - rx) / kx;
            rx = xsub(b[3], eps);
            ry = xadd(ry, xmul(ky, d));
            rz = xadd(rz, xmul(kz, d));
            cumds = xadd(cumds, d);
        }
        if (ry <= b[1])
        {
            if (ky <= 0.0) return false;
            double d = (b[1] - ry) / ky;
            rx = xadd(rx, xmul(kx, d));
            ry = xadd(b[1], eps);
            rz = xadd(rz, xmul(kz, d));
            cumds = xadd(cumds, d);
        }
        else if (ry >= b[4])
        {
            if (ky >= 0.0) return false;
            double d = (b[4] - ry) / ky;
            rx = xadd(rx, xmul(kx, d));
            ry = xsub(b[4], eps);
            rz = xadd(rz, xmul(kz, d));
            cumds = xadd(cumds, d);
        }
        if (rz <= b[2])
        {
            if (kz <= 0.0) return false;
            double d = (b[2] - rz) / kz;
            rx = xadd(rx, xmul(kx, d));
            ry = xadd(ry, xmul(ky, d));
            rz = xadd(b[2], eps);
            cumds = xadd(cumds, d);
        }
        else if (rz >= b[5])
        {
            if (kz >= 0.0) return false;
            double d = (b[5] - rz) / kz;
            rx = xadd(rx, xmul(kx, d));
            ry = xadd(ry, xmul(ky, d));
            rz = xsub(b[5], eps);
            cumds = xadd(cumds, d);
        }
        if (!boxContains(b, rx, ry, rz)) return false;
        m = -1;
        ds = cumds;
        state = GS_INSIDE;
        return true;
    }
};

// Box::diagonal (SKIRT/utils/Box.hpp:125-129) with separate roundings
SKG_D double boxDiagonal(const double* b)
{
    double dx = xsub(b[3], b[0]), dy = xsub(b[4], b[1]), dz = xsub(b[5], b[2]);
    return sqrt(xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz)));
}

// ---------------------------------------------------------------------------------------------
// Cartesian
// ---------------------------------------------------------------------------------------------
struct CartesianExact : GenBase
{
    static constexpr int kMinBlocks = 3;
    static constexpr int kRefillMin = 16;  // waiting lanes before a warp takes new tasks
    int i, j, k;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int = -1)
    {
        startRay(x, y, z, ux, uy, uz);
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        if (state == GS_UNKNOWN)
        {
            if (!moveInside(g.ext, xmul(1e-12, boxDiagonal(g.ext)))) return false;
            i = locateClip(g.xb, g.nx + 1, rx);
            j = locateClip(g.yb, g.ny + 1, ry);
            k = locateClip(g.zb, g.nz + 1, rz);
            if (ds > 0.) return true;
        }
        // state == inside
        int mm = k + g.nz * j + g.nz * g.ny * i;
        double xE = (kx < 0.0) ? g.xb[i] : g.xb[i + 1];
        double yE = (ky < 0.0) ? g.yb[j] : g.yb[j + 1];
        double zE = (kz < 0.0) ? g.zb[k] : g.zb[k + 1];
        double dsx = (fabs(kx) > 1e-15) ? xsub(xE, rx) / kx : DBL_MAX;
        double dsy = (fabs(ky) > 1e-15) ? xsub(yE, ry) / ky : DBL_MAX;
        double dsz = (fabs(kz) > 1e-15) ? xsub(zE, rz) / kz : DBL_MAX;
        if (dsx <= dsy && dsx <= dsz)
        {
            m = mm; ds = dsx;
            rx = xE;
            ry = xadd(ry, xmul(ky, dsx));
            rz = xadd(rz, xmul(kz, dsx));
            i += (kx < 0.0) ? -1 : 1;
            if (i >= g.nx || i < 0) state = GS_OUTSIDE;
        }
        else if (dsy < dsx && dsy <= dsz)
        {
            m = mm; ds = dsy;
            ry = yE;
            rx = xadd(rx, xmul(kx, dsy));
            rz = xadd(rz, xmul(kz, dsy));
            j += (ky < 0.0) ? -1 : 1;
            if (j >= g.ny || j < 0) state = GS_OUTSIDE;
        }
        else
        {
            m = mm; ds = dsz;
            rz = zE;
            rx = xadd(rx, xmul(kx, dsz));
            ry = xadd(ry, xmul(ky, dsz));
            k += (kz < 0.0) ? -1 : 1;
            if (k >= g.nz || k < 0) state = GS_OUTSIDE;
        }
        return true;
    }
};

// ---------------------------------------------------------------------------------------------
// Octree
// ---------------------------------------------------------------------------------------------
// TreeNode::leafChild from the root with OctTreeNode::child (TreeNode.cpp:66-76, OctTreeNode.cpp:37-42)
SKG_D int octreeLeafChild(const GridDev& g, double x, double y, double z)
{
    const double* b = g.tBounds;
    if (!GenBase::boxContains(b, x, y, z)) return -1;
    int node = 0;
    for (int guard = 0; guard < 64; ++guard)
    {
        int c0 = g.tChild[node];
        if (c0 < 0) return node;
        const double* cb = g.tBounds + 6 * static_cast<size_t>(c0);  // first child's rmax is the split point
        int l = (x < cb[3] ? 0 : 1) + (y < cb[4] ? 0 : 2) + (z < cb[5] ? 0 : 4);
        node = c0 + l;
    }
    return -1;
}

// AdaptiveMeshSnapshot::Node::leaf with Node::child (AdaptiveMeshSnapshot.cpp:103-145): the child
// holding the point is estimated by Box::cellIndices over the node's nx x ny x nz subdivision and
// corrected by one index per axis when the estimate does not contain the point. Returns -1 outside
// the root; -2 where the reference stops with "Can't locate the appropriate child node".
SKG_D int adaptiveLeaf(const GridDev& g, double x, double y, double z)
{
    if (!GenBase::boxContains(g.tBounds, x, y, z)) return -1;
    int node = 0;
    for (int guard = 0; guard < 256; ++guard)
    {
        const int* d = g.amDiv + 3 * static_cast<size_t>(node);
        int nx = d[0], ny = d[1], nz = d[2];
        if (nx == 0) return node;
        const double* b = g.tBounds + 6 * static_cast<size_t>(node);
        // Box::cellIndices (SKIRT/utils/Box.hpp:162-167)
        int i = max(0, min(nx - 1, static_cast<int>(xmul(static_cast<double>(nx), xsub(x, b[0])) / xsub(b[3], b[0]))));
        int j = max(0, min(ny - 1, static_cast<int>(xmul(static_cast<double>(ny), xsub(y, b[1])) / xsub(b[4], b[1]))));
        int k = max(0, min(nz - 1, static_cast<int>(xmul(static_cast<double>(nz), xsub(z, b[2])) / xsub(b[5], b[2]))));
        const int* kids = g.amChild + g.amChildBegin[node];
        int c = kids[(k * ny + j) * nx + i];
        const double* cb = g.tBounds + 6 * static_cast<size_t>(c);
        if (!GenBase::boxContains(cb, x, y, z))
        {
            if (x < cb[0]) i--;
            else if (x > cb[3]) i++;
            if (y < cb[1]) j--;
            else if (y > cb[4]) j++;
            if (z < cb[2]) k--;
            else if (z > cb[5]) k++;
            if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz) return -2;
            c = kids[(k * ny + j) * nx + i];
            if (!GenBase::boxContains(g.tBounds + 6 * static_cast<size_t>(c), x, y, z)) return -2;
        }
        node = c;
    }
    return -2;
}

// the leaf search of a tree walker: the octree's (TreeNode::leafChild) or the adaptive mesh's
template<bool Adaptive>
SKG_D int treeLeaf(const GridDev& g, double x, double y, double z)
{
    if (Adaptive)
    {
        int l = adaptiveLeaf(g, x, y, z);
        return l < 0 ? -1 : l;
    }
    return octreeLeafChild(g, x, y, z);
}

// TreeSpatialGrid::MySegmentGenerator::next (TreeSpatialGrid.cpp:143-228) and, with the adaptive
// leaf search, AdaptiveMeshSnapshot::MySegmentGenerator::next (AdaptiveMeshSnapshot.cpp:378-449):
// the same wall ties, step ds + eps, neighbour (list) then top-down search, nextafter escape.
template<bool Adaptive>
struct TreeExactT : GenBase
{
    static constexpr int kMinBlocks = 3;
    static constexpr int kRefillMin = 16;  // waiting lanes before a warp takes new tasks
    int node;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int = -1)
    {
        startRay(x, y, z, ux, uy, uz);
        node = -1;
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        if (state == GS_UNKNOWN)
        {
            if (!moveInside(g.ext, g.eps)) return false;
            node = treeLeaf<Adaptive>(g, rx, ry, rz);
            if (node < 0)
            {
                state = GS_OUTSIDE;
                return false;
            }
            if (ds > 0.) return true;
        }
        const double* b = g.tBounds + 6 * static_cast<size_t>(node);
        double xnext = (kx < 0.0) ? b[0] : b[3];
        double ynext = (ky < 0.0) ? b[1] : b[4];
        double znext = (kz < 0.0) ? b[2] : b[5];
        double dsx = (fabs(kx) > 1e-15) ? xsub(xnext, rx) / kx : DBL_MAX;
        double dsy = (fabs(ky) > 1e-15) ? xsub(ynext, ry) / ky : DBL_MAX;
        double dsz = (fabs(kz) > 1e-15) ? xsub(znext, rz) / kz : DBL_MAX;
        double d;
        int wall;
        if (dsx <= dsy && dsx <= dsz)
        {
            d = dsx;
            wall = (kx < 0.0) ? 0 : 1;
        }
        else if (dsy <= dsx && dsy <= dsz)
        {
            d = dsy;
            wall = (ky < 0.0) ? 2 : 3;
        }
        else
        {
            d = dsz;
            wall = (kz < 0.0) ? 4 : 5;
        }
        propagater(xadd(d, g.eps));
        m = g.tCell[node];
        ds = d;
        int old = node;
        // TreeNode::neighbor / Node::neighbor: the first neighbour across the wall (overlap-sorted
        // for the octree, the single most likely one for the adaptive mesh) containing r
        int nb = -1;
        int e0 = g.tNbBegin[6 * node + wall], e1 = g.tNbBegin[6 * node + wall + 1];
        for (int e = e0; e < e1; ++e)
        {
            int cand = g.tNb[e];
            if (boxContains(g.tBounds + 6 * static_cast<size_t>(cand), rx, ry, rz))
            {
                nb = cand;
                break;
            }
        }
        if (nb < 0) nb = treeLeaf<Adaptive>(g, rx, ry, rz);
        if (nb == old)
        {
            rx = nextafter(rx, (kx < 0.) ? -DBL_MAX : DBL_MAX);
            ry = nextafter(ry, (ky < 0.) ? -DBL_MAX : DBL_MAX);
            rz = nextafter(rz, (kz < 0.) ? -DBL_MAX : DBL_MAX);
            nb = treeLeaf<Adaptive>(g, rx, ry, rz);
        }
        node = nb;
        if (nb < 0 || nb == old) state = GS_OUTSIDE;
        return true;
    }
};

using OctreeExact = TreeExactT<false>;
using AdaptiveMeshExact = TreeExactT<true>;

// ---------------------------------------------------------------------------------------------
// Voronoi
// ---------------------------------------------------------------------------------------------
// Nearest site by an expanding search over a uniform block grid of sites. Returns the site with
// the smallest squared distance (VoronoiMeshSnapshot::cellIndex, VoronoiMeshSnapshot.cpp:1037-1067,
// selects the same site except for exactly equidistant ties).
SKG_D int voronoiCellIndex(const GridDev& g, double x, double y, double z)
{
    if (!GenBase::boxContains(g.ext, x, y, z)) return -1;
    const int n = g.vGridN;
    double wx = (g.ext[3] - g.ext[0]) / n, wy = (g.ext[4] - g.ext[1]) / n, wz = (g.ext[5] - g.ext[2]) / n;
    int bi = min(n - 1, max(0, static_cast<int>((x - g.ext[0]) / wx)));
    int bj = min(n - 1, max(0, static_cast<int>((y - g.ext[1]) / wy)));
    int bk = min(n - 1, max(0, static_cast<int>((z - g.ext[2]) / wz)));
    int best = -1;
    double bestd = DBL_MAX;
    double wmin = fmin(wx, fmin(wy, wz));
    for (int ring = 0; ring <= n; ++ring)
    {
        int i0 = bi - ring, i1 = bi + ring, j0 = bj - ring, j1 = bj + ring, k0 = bk - ring, k1 = bk + ring;
        for (int i = max(0, i0); i <= min(n - 1, i1); ++i)
            for (int j = max(0, j0); j <= min(n - 1, j1); ++j)
                for (int k = max(0, k0); k <= min(n - 1, k1); ++k)
                {
                    // only the shell of this ring
                    if (i != i0 && i != i1 && j != j0 && j != j1 && k != k0 && k != k1) continue;
                    int blk = (i * n + j) * n + k;
                    for (int e = g.vBlkBegin[blk]; e < g.vBlkBegin[blk + 1]; ++e)
                    {
                        int s = g.vBlkSites[e];
                        const double* p = g.vSites + 3 * static_cast<size_t>(s);
                        double dx = xsub(p[0], x), dy = xsub(p[1], y), dz = xsub(p[2], z);
                        double d2 = xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
                        if (d2 < bestd || (d2 == bestd && s < best))
                        {
                            bestd = d2;
                            best = s;
                        }
                    }
                }
        // every unsearched site is at least ring*wmin away from the query point
        if (best >= 0)
        {
            double reach = ring * wmin;
            if (reach * reach > bestd) break;
        }
    }
    return best;
}

struct VoronoiExact : GenBase
{
    static constexpr int kMinBlocks = 3;
    static constexpr int kRefillMin = 8;  // waiting lanes before a warp takes new tasks
    int mr;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int = -1)
    {
        startRay(x, y, z, ux, uy, uz);
        mr = -1;
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        if (state == GS_UNKNOWN)
        {
            if (!moveInside(g.ext, g.eps)) return false;
            mr = voronoiCellIndex(g, rx, ry, rz);
            if (mr < 0)
            {
                state = GS_OUTSIDE;
                return false;
            }
            if (ds > 0.) return true;
        }
        for (int guard = 0; guard < 1000; ++guard)
        {
            const double* pr = g.vSites + 3 * static_cast<size_t>(mr);
            double sq = DBL_MAX;
            const int NO_INDEX = -99;
            int mq = NO_INDEX;
            for (int e = g.vNbBegin[mr]; e < g.vNbBegin[mr + 1]; ++e)
            {
                int mi = g.vNb[e];
                double si = 0;
                if (mi >= 0)
                {
                    const double* pi = g.vSites + 3 * static_cast<size_t>(mi);
                    double nx = xsub(pi[0], pr[0]), ny = xsub(pi[1], pr[1]), nz = xsub(pi[2], pr[2]);
                    double ndotk = xdot3(nx, kx, ny, ky, nz, kz);
                    if (ndotk > 0)
                    {
                        double px = xmul(0.5, xadd(pi[0], pr[0]));
                        double py = xmul(0.5, xadd(pi[1], pr[1]));
                        double pz = xmul(0.5, xadd(pi[2], pr[2]));
                        si = xdot3(nx, xsub(px, rx), ny, xsub(py, ry), nz, xsub(pz, rz)) / ndotk;
                    }
                }
                else
                {
                    switch (mi)
                    {
                        case -1: si = xsub(g.ext[0], rx) / kx; break;
                        case -2: si = xsub(g.ext[3], rx) / kx; break;
                        case -3: si = xsub(g.ext[1], ry) / ky; break;
                        case -4: si = xsub(g.ext[4], ry) / ky; break;
                        case -5: si = xsub(g.ext[2], rz) / kz; break;
                        case -6: si = xsub(g.ext[5], rz) / kz; break;
                        default: si = 0; break;
                    }
                }
                if (si > 0 && si < sq)
                {
                    sq = si;
                    mq = mi;
                }
            }
            if (mq == NO_INDEX)
            {
                propagater(g.eps);
                mr = voronoiCellIndex(g, rx, ry, rz);
                if (mr < 0)
                {
                    state = GS_OUTSIDE;
                    return false;
                }
            }
            else
            {
                propagater(xadd(sq, g.eps));
                m = mr;
                ds = sq;
                mr = mq;
                if (mr < 0) state = GS_OUTSIDE;
                return true;
            }
        }
        state = GS_OUTSIDE;
        return false;
    }
};

// ---------------------------------------------------------------------------------------------
// Tetrahedral mesh
// ---------------------------------------------------------------------------------------------
SKG_D void teVertex(const GridDev& g, int t, int v, double& x, double& y, double& z)
{
    const double* p = g.teVerts + 3 * static_cast<size_t>(g.teTet[4 * static_cast<size_t>(t) + v]);
    x = p[0]; y = p[1]; z = p[2];
}

// Tetra::contains (TetraMeshSpatialGrid.cpp:114-138)
SKG_D bool teContains(const GridDev& g, int t, double x, double y, double z)
{
    if (!GenBase::boxContains(g.teBox + 6 * static_cast<size_t>(t), x, y, z)) return false;
    const double* nrm = g.teNormals + 12 * static_cast<size_t>(t);
    double vx, vy, vz;
    teVertex(g, t, 3, vx, vy, vz);
    for (int f = 0; f <= 2; ++f)
    {
        if (xdot3(xsub(vx, x), nrm[3 * f], xsub(vy, y), nrm[3 * f + 1], xsub(vz, z), nrm[3 * f + 2]) < 0) return false;
    }
    teVertex(g, t, 0, vx, vy, vz);
    if (xdot3(xsub(vx, x), nrm[9], xsub(vy, y), nrm[10], xsub(vz, z), nrm[11]) < 0.) return false;
    return true;
}

// TetraMeshSpatialGrid::cellIndex (TetraMeshSpatialGrid.cpp:615-622): first tetrahedron of the
// position's search block that contains it
SKG_D int tetraCellIndex(const GridDev& g, double x, double y, double z)
{
    if (!GenBase::boxContains(g.ext, x, y, z)) return -1;
    const int n = g.teGridN;
    int bi = min(n - 1, max(0, static_cast<int>(n * (x - g.ext[0]) / (g.ext[3] - g.ext[0]))));
    int bj = min(n - 1, max(0, static_cast<int>(n * (y - g.ext[1]) / (g.ext[4] - g.ext[1]))));
    int bk = min(n - 1, max(0, static_cast<int>(n * (z - g.ext[2]) / (g.ext[5] - g.ext[2]))));
    int blk = (bi * n + bj) * n + bk;
    for (int e = g.teBlkBegin[blk]; e < g.teBlkBegin[blk + 1]; ++e)
    {
        int t = g.teBlkTets[e];
        if (teContains(g, t, x, y, z)) return t;
    }
    return -1;
}

// clockwiseVertices (TetraMeshSpatialGrid.cpp:44-50)
SKG_D void clockwiseVertices(int face, int cv[3])
{
    cv[0] = (face + 3) % 4;
    cv[1] = (face + 2) % 4;
    cv[2] = (face + 1) % 4;
    if (face % 2 == 0)
    {
        int t = cv[0]; cv[0] = cv[2]; cv[2] = t;
    }
}

// Vec::cross (SKIRT/utils/Vec.hpp:73-76)
SKG_D void xcross(double ax, double ay, double az, double bx, double by, double bz, double& cx, double& cy, double& cz)
{
    cx = xsub(xmul(ay, bz), xmul(az, by));
    cy = xsub(xmul(az, bx), xmul(ax, bz));
    cz = xsub(xmul(ax, by), xmul(ay, bx));
}

// Tetra::findEnteringFace (TetraMeshSpatialGrid.cpp:87-112): the face of tetrahedron t the ray at
// (rx, ry, rz) with direction (kx, ky, kz) entered through, from Plucker products with its edges
SKG_D int teFindEnteringFace(const GridDev& g, int t, double rx, double ry, double rz, double kx, double ky, double kz)
{
    const int etable[6][2] = {{3, 2}, {1, 3}, {2, 1}, {3, 0}, {0, 2}, {1, 0}};
    int e = 0;
    for (int t1 = 0; t1 < 3; t1++)
    {
        double v1x, v1y, v1z;
        teVertex(g, t, t1, v1x, v1y, v1z);
        for (int t2 = t1 + 1; t2 < 4; t2++)
        {
            double v2x, v2y, v2z;
            teVertex(g, t, t2, v2x, v2y, v2z);
            double mx, my, mz;
            xcross(kx, ky, kz, xsub(rx, v1x), xsub(ry, v1y), xsub(rz, v1z), mx, my, mz);
            double prod = xdot3(mx, xsub(v2x, v1x), my, xsub(v2y, v1y), mz, xsub(v2z, v1z));
            if (prod != 0.) return prod < 0 ? etable[e][0] : etable[e][1];
            e++;
        }
    }
    return -1;
}

// The leaving face of tetrahedron t and the distance d to it, as one iteration of
// TetraMeshSpatialGrid::MySegmentGenerator::next decides them (TetraMeshSpatialGrid.cpp:720-785):
// the Plucker products of the ray with the edges of the entering face pick the leaving face; where a
// product is zero the smallest positive plane distance over the three other faces does. enteringFace
// is found first when it is -1. Returns -1 when no face lies ahead.
SKG_D int teLeavingFace(const GridDev& g, int t, int& enteringFace, double rx, double ry, double rz, double kx, double ky,
                        double kz, double& d)
{
    d = DBL_MAX;
    if (enteringFace == -1) enteringFace = teFindEnteringFace(g, t, rx, ry, rz, kx, ky, kz);
    if (enteringFace < 0) enteringFace = 0;  // degenerate direction: the plane fallback below decides
    double vex, vey, vez;
    teVertex(g, t, enteringFace, vex, vey, vez);
    double mx, my, mz;
    xcross(kx, ky, kz, xsub(rx, vex), xsub(ry, vey), xsub(rz, vez), mx, my, mz);
    int cv[3];
    clockwiseVertices(enteringFace, cv);
    double c0x, c0y, c0z;
    teVertex(g, t, cv[0], c0x, c0y, c0z);
    double prod0 = xdot3(mx, xsub(vex, c0x), my, xsub(vey, c0y), mz, xsub(vez, c0z));
    int clock0 = prod0 < 0;
    int i = clock0 ? 1 : 2;
    double cix, ciy, ciz;
    teVertex(g, t, cv[i], cix, ciy, ciz);
    double prodi = xdot3(mx, xsub(vex, cix), my, xsub(vey, ciy), mz, xsub(vez, ciz));
    int cclocki = prodi >= 0;
    const double* nrm = g.teNormals + 12 * static_cast<size_t>(t);
    int leavingFace = -1;
    if (prod0 == 0. || prodi == 0.)
    {
        for (int q = 0; q < 3; ++q)
        {
            int face = cv[q];
            const double* n = nrm + 3 * face;
            double ndotk = xdot3(n[0], kx, n[1], ky, n[2], kz);
            if (ndotk > 0)
            {
                double dq = xdot3(n[0], xsub(vex, rx), n[1], xsub(vey, ry), n[2], xsub(vez, rz)) / ndotk;
                if (dq < d)
                {
                    d = dq;
                    leavingFace = face;
                }
            }
        }
    }
    else
    {
        const int dtable[2][2] = {{1, 0}, {0, 2}};
        leavingFace = cv[dtable[clock0][cclocki]];
        const double* n = nrm + 3 * leavingFace;
        double ndotk = xdot3(n[0], kx, n[1], ky, n[2], kz);
        d = xdot3(n[0], xsub(vex, rx), n[1], xsub(vey, ry), n[2], xsub(vez, rz)) / ndotk;
    }
    return leavingFace;
}

struct TetraExact : GenBase
{
    static constexpr int kMinBlocks = 3;
    static constexpr int kRefillMin = 8;  // waiting lanes before a warp takes new tasks
    int mr;
    int enteringFace;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int = -1)
    {
        startRay(x, y, z, ux, uy, uz);
        mr = -1;
        enteringFace = -1;
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        if (state == GS_UNKNOWN)
        {
            if (!moveInside(g.ext, g.eps)) return false;
            mr = tetraCellIndex(g, rx, ry, rz);
            enteringFace = -1;
            if (mr == -1)
            {
                state = GS_OUTSIDE;
                return false;
            }
            if (ds > 0.) return true;
        }
        for (int guard = 0; guard < 1000; ++guard)
        {
            double d;
            int leavingFace = teLeavingFace(g, mr, enteringFace, rx, ry, rz, kx, ky, kz, d);
            if (leavingFace == -1 || d < g.eps)
            {
                propagater(g.eps);
                mr = tetraCellIndex(g, rx, ry, rz);
                if (mr < 0)
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                enteringFace = -1;
            }
            else
            {
                propagater(d);
                m = mr;
                ds = d;
                int nt = g.teNTet[4 * static_cast<size_t>(mr) + leavingFace];
                int nf = g.teNFace[4 * static_cast<size_t>(mr) + leavingFace];
                mr = nt;
                if (mr < 0)
                {
                    // the reference drops the final in-mesh segment when the path leaves the hull
                    state = GS_OUTSIDE;
                    return false;
                }
                enteringFace = nf;
                return true;
            }
        }
        state = GS_OUTSIDE;
        return false;
    }
};

// ---------------------------------------------------------------------------------------------
// 1D spherical grid (Sphere1DSpatialGrid::MySegmentGenerator::next, Sphere1DSpatialGrid.cpp):
// the radial shells are crossed inwards down to the shell of the impact parameter p, then
// outwards; each exit is at q_N = -/+ sqrt((r_N - p)(r_N + p)) along the ray, q measured from the
// projection of the origin. The position is not advanced: the generator tracks q.
// ---------------------------------------------------------------------------------------------
struct Sphere1DExact : GenBase
{
    static constexpr int kMinBlocks = 4;
    static constexpr int kRefillMin = 16;  // waiting lanes before a warp takes new tasks
    double q, p;
    int i, imin;
    bool inwards;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int = -1)
    {
        startRay(x, y, z, ux, uy, uz);
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        const double* rv = g.sRv;
        const int nr = g.sNr;
        if (state == GS_UNKNOWN)
        {
            double rmax = rv[nr], rmin = rv[0];
            double r = sqrt(xadd(xadd(xmul(rx, rx), xmul(ry, ry)), xmul(rz, rz)));
            q = xadd(xadd(xmul(rx, kx), xmul(ry, ky)), xmul(rz, kz));
            p = sqrt(xmul(xsub(r, q), xadd(r, q)));
            if (r > rmax)
            {
                if (q > 0. || p > rmax)
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                double qmax = -sqrt(xmul(xsub(rmax, p), xadd(rmax, p)));
                m = -1;
                ds = xsub(qmax, q);
                i = nr - 1;
                q = qmax;
                state = GS_INSIDE;
                imin = locateNR(rv, nr + 1, p);
                inwards = i > imin;
                return true;
            }
            else if (r < rmin)
            {
                double qmin = sqrt(xmul(xsub(rmin, p), xadd(rmin, p)));
                m = -1;
                ds = xsub(qmin, q);
                i = 0;
                q = qmin;
                state = GS_INSIDE;
                inwards = false;
                return true;
            }
            i = locateClip(rv, nr + 1, r);
            state = GS_INSIDE;
            inwards = false;
            if (q < 0.)
            {
                imin = locateNR(rv, nr + 1, p);
                if (i > imin) inwards = true;
            }
        }
        if (inwards)
        {
            double rN = rv[i];
            double qN = -sqrt(xmul(xsub(rN, p), xadd(rN, p)));
            m = i;
            ds = xsub(qN, q);
            i--;
            q = qN;
            if (i <= imin) inwards = false;
            return true;
        }
        double rN = rv[i + 1];
        double qN = sqrt(xmul(xsub(rN, p), xadd(rN, p)));
        m = i;
        ds = xsub(qN, q);
        i++;
        q = qN;
        if (i >= nr) state = GS_OUTSIDE;
        return true;
    }
};

// ---------------------------------------------------------------------------------------------
// 2D cylindrical grid (Cylinder2DSpatialGrid::MySegmentGenerator, Cylinder2DSpatialGrid.cpp:110-391):
// the ray in the meridional plane, with q its projection on the horizontal direction and p the
// horizontal impact parameter; each step exits either through the next cylinder (inwards down to the
// impact parameter's shell, then outwards) or through the next horizontal plane, whichever is
// nearer. Entry from outside by the generator's own moveInside (small inward nudges at the walls).
// ---------------------------------------------------------------------------------------------
struct Cylinder2DExact : GenBase
{
    static constexpr int kMinBlocks = 4;
    static constexpr int kRefillMin = 16;  // waiting lanes before a warp takes new tasks
    double cR, cz, kq, kzc, p, q;
    int i, k, imin;
    bool up, in;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int = -1)
    {
        startRay(x, y, z, ux, uy, uz);
        imin = -1;
    }

    SKG_D bool moveInsideCyl(const GridDev& g)
    {
        const double* Rv = g.cRv;
        const double* zv = g.czv;
        const int NR = g.cNR, Nz = g.cNz;
        cR = sqrt(xadd(xmul(rx, rx), xmul(ry, ry)));
        cz = rz;
        kq = sqrt(xadd(xmul(kx, kx), xmul(ky, ky)));
        kzc = kz;
        if (kq == 0.0) kq = 1e-20;
        if (kzc == 0.0) kzc = 1e-20;
        q = xadd(xmul(rx, kx), xmul(ry, ky)) / kq;
        double pp = xmul(xsub(cR, q), xadd(cR, q));
        p = sqrt(0. < pp ? pp : 0.);  // std::max(0., x)
        double Rmax = Rv[NR], zmin = zv[0], zmax = zv[Nz];
        m = -1;
        ds = 0.;
        state = GS_OUTSIDE;
        double cumds = 0.;
        if (cR >= Rmax)
        {
            if (q > 0.0 || p > Rmax) return false;
            double qmin = -sqrt(xmul(xsub(Rmax, p), xadd(Rmax, p)));
            double d = xsub(qmin, q) / kq;
            q = qmin;
            cR = xsub(Rmax, xmul(1e-8, xsub(Rv[NR], Rv[NR - 1])));
            cz = xadd(cz, xmul(kzc, d));
            cumds = xadd(cumds, d);
        }
        if (cz < zmin)
        {
            if (kzc <= 0.0) return false;
            double d = xsub(zmin, cz) / kzc;
            q = xadd(q, xmul(kq, d));
            cR = sqrt(xadd(xmul(p, p), xmul(q, q)));
            cz = xadd(zmin, xmul(1e-8, xsub(zv[1], zv[0])));
            cumds = xadd(cumds, d);
        }
        else if (cz > zmax)
        {
            if (kzc >= 0.0) return false;
            double d = xsub(zmax, cz) / kzc;
            q = xadd(q, xmul(kq, d));
            cR = sqrt(xadd(xmul(p, p), xmul(q, q)));
            cz = xsub(zmax, xmul(1e-8, xsub(zv[Nz], zv[Nz - 1])));
            cumds = xadd(cumds, d);
        }
        if (isinf(cR) || isnan(cR) || isinf(cz) || isnan(cz)) return false;
        if (cR >= Rmax || cz <= zmin || cz >= zmax) return false;
        m = -1;
        ds = cumds;
        state = GS_INSIDE;
        return true;
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        const double* Rv = g.cRv;
        const double* zv = g.czv;
        const int NR = g.cNR, Nz = g.cNz;
        if (state == GS_UNKNOWN)
        {
            if (!moveInsideCyl(g)) return false;
            i = locateNR(Rv, NR + 1, cR);
            k = locateClip(zv, Nz + 1, cz);
            up = kzc >= 0.;
            in = false;
            if (q < 0.)
            {
                imin = locateNR(Rv, NR + 1, p);
                if (i > imin) in = true;
            }
            if (ds > 0.) return true;
        }
        double RN = in ? Rv[i] : Rv[i + 1];
        double w = sqrt(xmul(xsub(RN, p), xadd(RN, p)));
        double qN = in ? -w : w;
        double zN = up ? zv[k + 1] : zv[k];
        int mc = i < 0 ? -1 : k + Nz * i;  // Cylinder2DSpatialGrid::index
        double dsq = xsub(qN, q) / kq;
        double dsz = xsub(zN, cz) / kzc;
        if (dsq < dsz)
        {
            m = mc;
            ds = dsq;
            if (in)
            {
                i--;
                q = qN;
                cz = xadd(cz, xmul(kzc, dsq));
                if (i <= imin) in = false;
            }
            else
            {
                i++;
                if (i >= NR)
                    state = GS_OUTSIDE;
                else
                {
                    q = qN;
                    cz = xadd(cz, xmul(kzc, dsq));
                }
            }
        }
        else
        {
            m = mc;
            ds = dsz;
            k += up ? 1 : -1;
            if (up ? k >= Nz : k < 0)
                state = GS_OUTSIDE;
            else
            {
                q = xadd(q, xmul(kq, dsz));
                cz = zN;
            }
        }
        return true;
    }
};

// ---------------------------------------------------------------------------------------------
// 2D spherical grid (Sphere2DSpatialGrid::MySegmentGenerator::next, Sphere2DSpatialGrid.cpp:147-290):
// from the current position the nearest positive intersection with the cell's two spheres and two
// cones wins; the position advances by the segment plus eps = 1e-11 r_max and the cell indices
// follow the winning boundary. Sphere and cone intersections by the reference's quadratic
// solvers (Quadratic.hpp:44-68, Sphere2DSpatialGrid.cpp:118-142).
// ---------------------------------------------------------------------------------------------
SKG_D double quadSps(double b, double c)
{
    if (xmul(b, b) > c)
    {
        if (b > 0.)
        {
            if (c < 0.)
            {
                double x1 = xsub(-b, sqrt(xsub(xmul(b, b), c)));
                return c / x1;
            }
        }
        else
        {
            double x2 = xadd(-b, sqrt(xsub(xmul(b, b), c)));
            if (c > 0.)
            {
                double x1 = c / x2;
                if (x1 < x2) return x1;
            }
            return x2;
        }
    }
    return 0.;
}

SKG_D double quadSps3(double a, double b, double c)
{
    if (fabs(a) > 1e-9) return quadSps(b / a, c / a);
    double x = xmul(-0.5, c) / b;
    if (x > 0.) return x;
    return 0.;
}

struct Sphere2DExact : GenBase
{
    static constexpr int kMinBlocks = 3;
    static constexpr int kRefillMin = 16;  // waiting lanes before a warp takes new tasks
    int i, j;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int = -1)
    {
        startRay(x, y, z, ux, uy, uz);
    }

    SKG_D double dotRK() const { return xadd(xadd(xmul(rx, kx), xmul(ry, ky)), xmul(rz, kz)); }
    SKG_D double norm2R() const { return xadd(xadd(xmul(rx, rx), xmul(ry, ry)), xmul(rz, rz)); }
    SKG_D double sphere(double r) const { return quadSps(dotRK(), xsub(norm2R(), xmul(r, r))); }
    SKG_D double cone(double c) const
    {
        if (c == 0.) return -rz / kz;
        double cc = xmul(c, c);
        return quadSps3(xsub(cc, xmul(kz, kz)), xsub(xmul(cc, dotRK()), xmul(rz, kz)), xsub(xmul(cc, norm2R()), xmul(rz, rz)));
    }

    // setCellIndices (Sphere2DSpatialGrid.cpp:160-167) with Position::spherical
    SKG_D bool indices(const GridDev& g)
    {
        double radius = sqrt(norm2R());
        double theta = radius == 0 ? 0. : acos(rz / radius);
        i = locateNR(g.s2r, g.s2Nr + 1, radius);
        j = locateClip(g.s2t, g.s2Nt + 1, theta);
        return i < g.s2Nr;
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        const double* rv = g.s2r;
        const double* cv = g.s2c;
        const int Nr = g.s2Nr, Nt = g.s2Nt;
        const double eps = xmul(1e-11, rv[Nr]);
        if (state == GS_UNKNOWN)
        {
            double rn = sqrt(norm2R());
            if (rn > rv[Nr])
            {
                double d = sphere(rv[Nr]);
                if (d <= 0.)
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                propagater(xadd(d, eps));
                if (!indices(g))
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                m = -1;
                ds = d;
                state = GS_INSIDE;
                return true;
            }
            if (rn < eps) propagater(eps);
            if (!indices(g))
            {
                state = GS_OUTSIDE;
                return false;
            }
            state = GS_INSIDE;
        }
        for (int guard = 0; guard < 1000; ++guard)
        {
            int icur = i, jcur = j;
            double d = DBL_MAX;
            if (icur > 0 || (icur == 0 && rv[0] > 0.))
            {
                double t = sphere(rv[icur]);
                if (t > 0 && t < d)
                {
                    d = t;
                    i = icur - 1;
                    j = jcur;
                }
            }
            {
                double t = sphere(rv[icur + 1]);
                if (t > 0 && t < d)
                {
                    d = t;
                    i = icur + 1;
                    j = jcur;
                }
            }
            if (jcur > 0)
            {
                double t = cone(cv[jcur]);
                if (t > 0 && t < d)
                {
                    d = t;
                    i = icur;
                    j = jcur - 1;
                }
            }
            if (jcur < Nt - 1)
            {
                double t = cone(cv[jcur + 1]);
                if (t > 0 && t < d)
                {
                    d = t;
                    i = icur;
                    j = jcur + 1;
                }
            }
            if (i != icur || j != jcur)
            {
                m = jcur + Nt * icur;  // Sphere2DSpatialGrid::index (negative inside r_0)
                ds = d;
                propagater(xadd(d, eps));
                if (i >= Nr) state = GS_OUTSIDE;
                return true;
            }
            propagater(eps);
            if (!indices(g))
            {
                state = GS_OUTSIDE;
                return false;
            }
        }
        state = GS_OUTSIDE;
        return false;
    }
};

// ---------------------------------------------------------------------------------------------
// 3D spherical grid (Sphere3DSpatialGrid::MySegmentGenerator, Sphere3DSpatialGrid.cpp:160-370):
// the nearest positive intersection of the cell's two spheres, two cones and two meridional planes
// (EPS = 1e-12, :20); inside the (possibly artificial) inner hole one empty step to the hole's
// sphere, after which the azimuth bin is re-derived from the position.
// ---------------------------------------------------------------------------------------------
struct Sphere3DExact : GenBase
{
    static constexpr int kMinBlocks = 3;
    static constexpr int kRefillMin = 16;  // waiting lanes before a warp takes new tasks
    int i, j, k;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int = -1)
    {
        startRay(x, y, z, ux, uy, uz);
    }

    SKG_D double dotRK() const { return xadd(xadd(xmul(rx, kx), xmul(ry, ky)), xmul(rz, kz)); }
    SKG_D double norm2R() const { return xadd(xadd(xmul(rx, rx), xmul(ry, ry)), xmul(rz, rz)); }
    SKG_D double sphere(double r) const { return quadSps(dotRK(), xsub(norm2R(), xmul(r, r))); }
    SKG_D static double sps3(double a, double b, double c)
    {
        if (fabs(a) > 1e-12) return quadSps(b / a, c / a);
        double x = xmul(-0.5, c) / b;
        if (x > 0.) return x;
        return 0.;
    }
    SKG_D double cone(double c) const
    {
        if (c == 0.) return -rz / kz;
        double cc = xmul(c, c);
        return sps3(xsub(cc, xmul(kz, kz)), xsub(xmul(cc, dotRK()), xmul(rz, kz)), xsub(xmul(cc, norm2R()), xmul(rz, rz)));
    }
    SKG_D double plane(double sn, double cs) const
    {
        double q = xsub(xmul(kx, sn), xmul(ky, cs));
        if (fabs(q) < 1e-12) return 0.;
        return -xsub(xmul(rx, sn), xmul(ry, cs)) / q;
    }
    // setCellIndices with Position::spherical (Sphere3DSpatialGrid.cpp:175-183)
    SKG_D bool indices(const GridDev& g)
    {
        double radius = sqrt(norm2R());
        double theta = 0., phi = 0.;
        if (radius != 0)
        {
            theta = acos(rz / radius);
            phi = atan2(ry, rx);
        }
        i = locateNR(g.s3r, g.s3Nr + 1, radius);
        j = locateClip(g.s3t, g.s3Nt + 1, theta);
        k = locateClip(g.s3p, g.s3Np + 1, phi);
        return i < g.s3Nr;
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        const double* rv = g.s3r;
        const int Nr = g.s3Nr, Nt = g.s3Nt, Np = g.s3Np;
        const double eps = g.s3eps;
        if (state == GS_UNKNOWN)
        {
            double rn = sqrt(norm2R());
            if (rn > rv[Nr])
            {
                double d = sphere(rv[Nr]);
                if (d <= 0.)
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                propagater(xadd(d, eps));
                if (!indices(g))
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                m = -1;
                ds = d;
                state = GS_INSIDE;
                return true;
            }
            if (!indices(g))
            {
                state = GS_OUTSIDE;
                return false;
            }
            state = GS_INSIDE;
        }
        if (i >= 0)
        {
            int icur = i, jcur = j, kcur = k;
            double d = DBL_MAX;
            {
                double t = sphere(rv[icur]);
                if (t > 0 && t < d) { d = t; i = icur - 1; j = jcur; k = kcur; }
            }
            {
                double t = sphere(rv[icur + 1]);
                if (t > 0 && t < d) { d = t; i = icur + 1; j = jcur; k = kcur; }
            }
            if (jcur > 0)
            {
                double t = cone(g.s3c[jcur]);
                if (t > 0 && t < d) { d = t; i = icur; j = jcur - 1; k = kcur; }
            }
            if (jcur < Nt - 1)
            {
                double t = cone(g.s3c[jcur + 1]);
                if (t > 0 && t < d) { d = t; i = icur; j = jcur + 1; k = kcur; }
            }
            {
                double t = plane(g.s3s[kcur], g.s3k[kcur]);
                if (t > 0. && t < d) { d = t; i = icur; j = jcur; k = kcur > 0 ? kcur - 1 : Np - 1; }
            }
            {
                double t = plane(g.s3s[kcur + 1], g.s3k[kcur + 1]);
                if (t > 0. && t < d) { d = t; i = icur; j = jcur; k = (kcur + 1) % Np; }
            }
            if (d == DBL_MAX)
            {
                state = GS_OUTSIDE;
                return false;
            }
            m = kcur + (jcur + icur * Nt) * Np;  // Sphere3DSpatialGrid::index
            ds = d;
            propagater(xadd(d, eps));
            if (i >= Nr) state = GS_OUTSIDE;
            return true;
        }
        double d = sphere(rv[0]);
        if (d <= 0.)
        {
            state = GS_OUTSIDE;
            return false;
        }
        m = -1;
        ds = d;
        propagater(xadd(d, eps));
        if (!indices(g))
        {
            state = GS_OUTSIDE;
            return false;
        }
        return true;
    }
};

// ---------------------------------------------------------------------------------------------
// 3D cylindrical grid (Cylinder3DSpatialGrid::MySegmentGenerator, Cylinder3DSpatialGrid.cpp:180-440):
// the nearest positive intersection of the cell's two cylinders, two meridional planes and two
// horizontal planes (EPS = 1e-12, :19); entry from outside by steps to the outer cylinder and the
// bounding plane; in the artificial inner hole a segment of the hole's azimuth bin up to the hole
// cylinder or a horizontal plane, in a real hole one empty step to the hole cylinder.
// ---------------------------------------------------------------------------------------------
// NR::locateFail (SKIRT/utils/NR.hpp:186-191): -1 outside [xv[0], xv[n - 1]]
SKG_D int locateFailNR(const double* xv, int n, double x)
{
    if (x > xv[n - 1]) return -1;
    int jl = -1, ju = n - 1;
    while (ju - jl > 1)
    {
        int jm = (ju + jl) >> 1;
        if (x < xv[jm])
            ju = jm;
        else
            jl = jm;
    }
    return jl;
}

struct Cylinder3DExact : GenBase
{
    static constexpr int kMinBlocks = 3;
    static constexpr int kRefillMin = 16;  // waiting lanes before a warp takes new tasks
    double kq2;
    int i, j, k;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int = -1)
    {
        startRay(x, y, z, ux, uy, uz);
    }

    SKG_D double cyl(const GridDev& g, int ii) const
    {
        if (fabs(kq2) < 1e-12) return 0.;
        double b = xadd(xmul(rx, kx), xmul(ry, ky));
        double c = xsub(xadd(xmul(rx, rx), xmul(ry, ry)), xmul(g.c3r[ii], g.c3r[ii]));
        return quadSps(b / kq2, c / kq2);
    }
    SKG_D double meridional(const GridDev& g, int jj) const
    {
        double sn = g.c3s[jj], cs = g.c3k[jj];
        double q = xsub(xmul(kx, sn), xmul(ky, cs));
        if (fabs(q) < 1e-12) return 0.;
        return -xsub(xmul(rx, sn), xmul(ry, cs)) / q;
    }
    SKG_D double horizontal(const GridDev& g, int kk) const
    {
        if (fabs(kz) < 1e-12) return 0.;
        return xsub(g.c3z[kk], rz) / kz;
    }
    // setCellIndices with Position::cylindrical (Cylinder3DSpatialGrid.cpp:195-203)
    SKG_D bool indices(const GridDev& g)
    {
        double R = sqrt(xadd(xmul(rx, rx), xmul(ry, ry)));
        double phi = atan2(ry, rx);
        i = locateNR(g.c3r, g.c3Nr + 1, R);
        j = locateClip(g.c3p, g.c3Np + 1, phi);
        k = locateFailNR(g.c3z, g.c3Nz + 1, rz);
        return i < g.c3Nr && k >= 0;
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        const int NR = g.c3Nr, Np = g.c3Np, Nz = g.c3Nz;
        const double eps = g.c3eps;
        if (state == GS_UNKNOWN)
        {
            kq2 = xadd(xmul(kx, kx), xmul(ky, ky));
            double cumds = 0.;
            double R = sqrt(xadd(xmul(rx, rx), xmul(ry, ry)));
            if (R > g.c3r[NR])
            {
                double d = cyl(g, NR);
                if (d <= 0.)
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                propagater(xadd(d, eps));
                cumds = xadd(cumds, d);
            }
            if (rz < g.c3z[0])
            {
                double d = horizontal(g, 0);
                if (d <= 0.)
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                propagater(xadd(d, eps));
                cumds = xadd(cumds, d);
            }
            else if (rz > g.c3z[Nz])
            {
                double d = horizontal(g, Nz);
                if (d <= 0.)
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                propagater(xadd(d, eps));
                cumds = xadd(cumds, d);
            }
            if (!indices(g))
            {
                state = GS_OUTSIDE;
                return false;
            }
            state = GS_INSIDE;
            if (cumds != 0.)
            {
                m = -1;
                ds = cumds;
                return true;
            }
        }
        if (i >= 0)
        {
            int icur = i, jcur = j, kcur = k;
            double d = DBL_MAX, t;
            t = cyl(g, icur);
            if (t > 0. && t < d) { d = t; i = icur - 1; j = jcur; k = kcur; }
            t = cyl(g, icur + 1);
            if (t > 0. && t < d) { d = t; i = icur + 1; j = jcur; k = kcur; }
            t = meridional(g, jcur);
            if (t > 0. && t < d) { d = t; i = icur; j = jcur > 0 ? jcur - 1 : Np - 1; k = kcur; }
            t = meridional(g, jcur + 1);
            if (t > 0. && t < d) { d = t; i = icur; j = (jcur + 1) % Np; k = kcur; }
            t = horizontal(g, kcur);
            if (t > 0 && t < d) { d = t; i = icur; j = jcur; k = kcur - 1; }
            t = horizontal(g, kcur + 1);
            if (t > 0. && t < d) { d = t; i = icur; j = jcur; k = kcur + 1; }
            if (d == DBL_MAX)
            {
                state = GS_OUTSIDE;
                return false;
            }
            m = kcur + (jcur + icur * Np) * Nz;  // Cylinder3DSpatialGrid::index
            ds = d;
            propagater(xadd(d, eps));
            if (i >= NR || k < 0 || k >= Nz) state = GS_OUTSIDE;
            return true;
        }
        if (!g.c3Hole)
        {
            int kcur = k;
            double d = DBL_MAX, t;
            t = cyl(g, 0);
            if (t > 0. && t < d) d = t;
            t = horizontal(g, kcur);
            if (t > 0 && t < d) { d = t; k = kcur - 1; }
            t = horizontal(g, kcur + 1);
            if (t > 0. && t < d) { d = t; k = kcur + 1; }
            if (d == DBL_MAX)
            {
                state = GS_OUTSIDE;
                return false;
            }
            m = kcur + j * Nz;  // index(0, j, kcur)
            ds = d;
            propagater(xadd(d, eps));
            if (k == kcur)
            {
                if (!indices(g))
                {
                    state = GS_OUTSIDE;
                    return false;
                }
            }
            else if (k < 0 || k >= Nz)
                state = GS_OUTSIDE;
            return true;
        }
        double d = cyl(g, 0);
        if (d <= 0.)
        {
            state = GS_OUTSIDE;
            return false;
        }
        m = -1;
        ds = d;
        propagater(xadd(d, eps));
        if (!indices(g))
        {
            state = GS_OUTSIDE;
            return false;
        }
        return true;
    }
};

}  // namespace skg
