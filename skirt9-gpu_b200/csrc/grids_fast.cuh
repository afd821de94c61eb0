// Production walkers. The Cartesian and octree walkers follow the reference generators' FP64
// operation order exactly (every wall distance, position update and containment test), so their
// cell sequences and segment lengths equal the reference's bit for bit; what makes them fast is the
// data layout and the division: a wall distance is the correctly rounded quotient from the ray's
// precomputed reciprocal direction (qdiv, three FP64 operations), and the octree walker reads
// 64-byte leaf records with exact FP64 walls from small per-axis lattice tables. Optical depth,
// path length and radiation-field factors accumulate in FP32 (Acc); tallies stay FP64. The Voronoi
// and tetrahedral walkers below keep FP32 face distances with FP64 re-decisions.
#pragma once

#include <type_traits>

#include "grids.cuh"

namespace skg {

// 1 / k rounded to nearest for |k| > 1e-15 (the reference's threshold for a usable direction
// component), 0 otherwise
SKG_D double recipDir(double k) { return fabs(k) > 1e-15 ? 1.0 / k : 0.0; }

// the reference's wall distance (wall - r) / k, or DBL_MAX for |k| <= 1e-15
SKG_D double wallDist(double wall, double r, double k, double ik)
{
    return fabs(k) > 1e-15 ? qdiv(xsub(wall, r), k, ik) : DBL_MAX;
}

// ---------------------------------------------------------------------------------------------
// Cartesian grid, production (CartesianSpatialGrid::MySegmentGenerator::next,
// CartesianSpatialGrid.cpp:77-155): the reference's steps with the quotient from the reciprocal
// direction; border arrays stay in L1.
// ---------------------------------------------------------------------------------------------
struct CartesianFast : GenBase
{
    using Acc = float;
    static constexpr int kMinBlocks = 4;
    static constexpr int kRefillMin = 16;  // waiting lanes before a warp takes new tasks
    int i, j, k;
    double ikx, iky, ikz;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int = -1)
    {
        startRay(x, y, z, ux, uy, uz);
        ikx = recipDir(ux);
        iky = recipDir(uy);
        ikz = recipDir(uz);
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
        int mm = k + g.nz * j + g.nz * g.ny * i;
        double xE = (kx < 0.0) ? __ldg(g.xb + i) : __ldg(g.xb + i + 1);
        double yE = (ky < 0.0) ? __ldg(g.yb + j) : __ldg(g.yb + j + 1);
        double zE = (kz < 0.0) ? __ldg(g.zb + k) : __ldg(g.zb + k + 1);
        double dsx = wallDist(xE, rx, kx, ikx);
        double dsy = wallDist(yE, ry, ky, iky);
        double dsz = wallDist(zE, rz, kz, ikz);
        m = mm;
        if (dsx <= dsy && dsx <= dsz)
        {
            ds = dsx;
            rx = xE;
            ry = xadd(ry, xmul(ky, dsx));
            rz = xadd(rz, xmul(kz, dsx));
            i += (kx < 0.0) ? -1 : 1;
            if (i >= g.nx || i < 0) state = GS_OUTSIDE;
        }
        else if (dsy < dsx && dsy <= dsz)
        {
            ds = dsy;
            ry = yE;
            rx = xadd(rx, xmul(kx, dsy));
            rz = xadd(rz, xmul(kz, dsy));
            j += (ky < 0.0) ? -1 : 1;
            if (j >= g.ny || j < 0) state = GS_OUTSIDE;
        }
        else
        {
            ds = dsz;
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
// Octree, production (TreeSpatialGrid::MySegmentGenerator::next, TreeSpatialGrid.cpp:143-228,
// TreeNode::neighbor, TreeNode.cpp:103-112). The reference takes the first neighbour across the
// exit wall, in overlap order, whose closed box contains the new position (Box::contains). Here:
//  - a wall with a single positive-overlap neighbour: that neighbour's face covers the whole wall,
//    and since entering the current cell (whose closed box held the position) the position has only
//    moved towards the cell's exit walls; so the neighbour contains it exactly when it lies at or
//    beyond the crossed wall and not beyond the other two exit walls: comparisons with the FP64
//    exit walls held in registers (on the crossed axis the neighbour's far wall is at least one
//    finest cell away, far beyond the eps step);
//  - a wall with several neighbours, or a position past a corner: each candidate's six FP64 walls
//    from the FP64 lattice tables, indexed by its record's 16-bit wall indices;
//  - otherwise the reference's complete procedure on the FP64 node arrays: the wall's full neighbour
//    list, the top-down search, the nextafter escape.
// Entering a cell reads its exit walls from the lattice tables. A start in a known cell (a
// scattering event's interaction cell) skips the top-down search when the top-down search would
// return that cell (half-open bounds).
// ---------------------------------------------------------------------------------------------
#ifndef SKG_OCTREE_MIN_BLOCKS
#define SKG_OCTREE_MIN_BLOCKS 4
#endif

struct OctreeRec : GenBase
{
    using Acc = float;
    static constexpr int kMinBlocks = SKG_OCTREE_MIN_BLOCKS;
    static constexpr int kRefillMin = 16;  // waiting lanes before a warp takes new tasks
    double xE, yE, zE;                     // exit walls of the current cell in the direction of travel

    // the ray's reciprocal direction lives in a per-thread shared-memory slot (blocks of at most
    // 256 threads), which keeps the walker's state within the registers of four resident blocks
    SKG_D static double* recip()
    {
        __shared__ double slots[3][256];
        return &slots[0][threadIdx.x];
    }
    int cell;                              // the current cell; before the first step the start cell when
                                           // the caller knows it (an interaction cell), else -1
    float cellDens, segDens;               // density of the current cell / of the segment just returned

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int h = -1)
    {
        startRay(x, y, z, ux, uy, uz);
        double* ik = recip();
        ik[0] = recipDir(ux);
        ik[256] = recipDir(uy);
        ik[512] = recipDir(uz);
        cell = h;
    }

    SKG_D double density(const double*) const { return static_cast<double>(segDens); }

    SKG_D static double wall(const GridDev& g, int axis, unsigned idx)
    {
        return __ldg(g.tWall + axis * g.tWallN + idx);
    }

    SKG_D static unsigned lo(int w) { return static_cast<unsigned>(w) & 0xFFFFu; }
    SKG_D static unsigned hi(int w) { return static_cast<unsigned>(w) >> 16; }

    // the six FP64 walls of the cell with record word w0
    SKG_D static void walls(const GridDev& g, int4 w0, double& x0, double& x1, double& y0, double& y1, double& z0,
                            double& z1)
    {
        x0 = wall(g, 0, lo(w0.x));
        x1 = wall(g, 0, hi(w0.x));
        y0 = wall(g, 1, lo(w0.y));
        y1 = wall(g, 1, hi(w0.y));
        z0 = wall(g, 2, lo(w0.z));
        z1 = wall(g, 2, hi(w0.z));
    }

    SKG_D void become(int c, float dens, double x0, double x1, double y0, double y1, double z0, double z1)
    {
        cell = c;
        cellDens = dens;
        xE = kx < 0.0 ? x0 : x1;
        yE = ky < 0.0 ? y0 : y1;
        zE = kz < 0.0 ? z0 : z1;
    }

    // enters c, whose closed box is known to hold the position
    SKG_D void enter(const GridDev& g, int c)
    {
        int4 w0 = __ldg(g.tRec + 4 * static_cast<size_t>(c));
        cell = c;
        cellDens = __int_as_float(w0.w);
        xE = wall(g, 0, kx < 0.0 ? lo(w0.x) : hi(w0.x));
        yE = wall(g, 1, ky < 0.0 ? lo(w0.y) : hi(w0.y));
        zE = wall(g, 2, kz < 0.0 ? lo(w0.z) : hi(w0.z));
    }

    // Box::contains (closed bounds) of cell c; on success c becomes the current cell
    SKG_D bool tryEnter(const GridDev& g, int c)
    {
        int4 w0 = __ldg(g.tRec + 4 * static_cast<size_t>(c));
        double x0, x1, y0, y1, z0, z1;
        walls(g, w0, x0, x1, y0, y1, z0, z1);
        bool in = rx >= x0 && rx <= x1 && ry >= y0 && ry <= y1 && rz >= z0 && rz <= z1;
        if (in) become(c, __int_as_float(w0.w), x0, x1, y0, y1, z0, z1);
        return in;
    }

    // the known start cell, if the top-down search (TreeNode::leafChild with OctTreeNode::child:
    // lower half for coordinates below the centre) would return it: lo <= r < hi per axis, or r on
    // the domain's upper wall
    SKG_D bool tryHint(const GridDev& g, int c)
    {
        int4 w0 = __ldg(g.tRec + 4 * static_cast<size_t>(c));
        double x0, x1, y0, y1, z0, z1;
        walls(g, w0, x0, x1, y0, y1, z0, z1);
        bool in = rx >= x0 && (rx < x1 || (rx == x1 && x1 == g.ext[3])) && ry >= y0
                  && (ry < y1 || (ry == y1 && y1 == g.ext[4])) && rz >= z0 && (rz < z1 || (rz == z1 && z1 == g.ext[5]));
        if (in) become(c, __int_as_float(w0.w), x0, x1, y0, y1, z0, z1);
        return in;
    }

    SKG_D static int locate(const GridDev& g, double x, double y, double z)
    {
        int n = octreeLeafChild(g, x, y, z);
        return n < 0 ? -1 : g.tCell[n];
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        if (state == GS_UNKNOWN)
        {
            if (!moveInside(g.ext, g.eps)) return false;
            if (!(cell >= 0 && ds == 0. && tryHint(g, cell)))
            {
                int c = locate(g, rx, ry, rz);
                if (c < 0)
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                enter(g, c);
            }
            if (ds > 0.) return true;
        }
        const double* ik = recip();
        double dsx = wallDist(xE, rx, kx, ik[0]);
        double dsy = wallDist(yE, ry, ky, ik[256]);
        double dsz = wallDist(zE, rz, kz, ik[512]);
        bool ax = dsx <= dsy && dsx <= dsz;
        bool ay = !ax && dsy <= dsx && dsy <= dsz;
        int axis = ax ? 0 : (ay ? 1 : 2);
        double d = ax ? dsx : (ay ? dsy : dsz);
        propagater(xadd(d, g.eps));
        m = cell;
        ds = d;
        segDens = cellDens;
        const int old = cell;
        // exit wall index: 2 * axis, +1 when the ray moves towards the upper wall
        const int wl = 2 * axis + ((axis == 0 ? kx : (axis == 1 ? ky : kz)) < 0.0 ? 0 : 1);
        const int* R = reinterpret_cast<const int*>(g.tRec + 4 * static_cast<size_t>(old));
        int one = __ldg(R + 8 + wl);
        // single neighbour: at or beyond the crossed exit wall, within the other two (branch free)
        bool bxE = kx < 0.0 ? rx <= xE : rx >= xE, wxE = kx < 0.0 ? rx >= xE : rx <= xE;
        bool byE = ky < 0.0 ? ry <= yE : ry >= yE, wyE = ky < 0.0 ? ry >= yE : ry <= yE;
        bool bzE = kz < 0.0 ? rz <= zE : rz >= zE, wzE = kz < 0.0 ? rz >= zE : rz <= zE;
        bool inOne = ax ? (bxE && wyE && wzE) : (ay ? (byE && wxE && wzE) : (bzE && wxE && wyE));
        bool found = false;
        if (one >= 0 && inOne)
        {
            enter(g, one);
            found = true;
        }
        else if (one >= 0)
        {
            found = tryEnter(g, one);
        }
        else if (one == -2)
        {
            unsigned long long cnt = (static_cast<unsigned long long>(static_cast<unsigned>(__ldg(R + 6))) << 32)
                                     | static_cast<unsigned>(__ldg(R + 5));
            if (cnt != ~0ULL)
            {
                int base = __ldg(R + 4);
                int e0 = base + static_cast<int>((cnt >> (9 * wl)) & 511);
                int e1 = base + static_cast<int>((cnt >> (9 * (wl + 1))) & 511);
                for (int e = e0; e < e1 && !found; ++e) found = tryEnter(g, __ldg(g.tLeafNb + e));
            }
        }
        if (!found)
        {
            // the reference's complete procedure on the FP64 node arrays: the wall's full neighbour
            // list in overlap order, the top-down search, the nextafter escape
            int node = __ldg(R + 7);
            int nb = -1;
            int e1 = g.tNbBegin[6 * node + wl + 1];
            for (int e = g.tNbBegin[6 * node + wl]; e < e1; ++e)
            {
                int cand = g.tNb[e];
                if (boxContains(g.tBounds + 6 * static_cast<size_t>(cand), rx, ry, rz))
                {
                    nb = cand;
                    break;
                }
            }
            if (nb < 0) nb = octreeLeafChild(g, rx, ry, rz);
            if (nb == node)
            {
                rx = nextafter(rx, (kx < 0.) ? -DBL_MAX : DBL_MAX);
                ry = nextafter(ry, (ky < 0.) ? -DBL_MAX : DBL_MAX);
                rz = nextafter(rz, (kz < 0.) ? -DBL_MAX : DBL_MAX);
                nb = octreeLeafChild(g, rx, ry, rz);
            }
            if (nb < 0 || nb == node)
                state = GS_OUTSIDE;
            else
                enter(g, g.tCell[nb]);
        }
        return true;
    }
};

// Octree, production precision for trees that are not a lattice of depth <= 15 (no leaf records):
// the FP64 node walker with FP32 accumulators
struct OctreeNodeFast : OctreeExact
{
    using Acc = float;
};

// Adaptive mesh, production: the reference-order FP64 walk (single neighbour per wall, top-down
// fallback) with FP32 accumulators
struct AdaptiveMeshFast : AdaptiveMeshExact
{
    using Acc = float;
};

// Nearest site of a point by a greedy walk on the neighbour graph (the Delaunay graph of the sites,
// on which the walk towards ever nearer sites ends at the nearest one), starting from the
// representative site of the point's block in the site-search grid. -1 outside the domain.
SKG_D int voronoiLocate(const GridDev& g, double x, double y, double z)
{
    if (!GenBase::boxContains(g.ext, x, y, z)) return -1;
    const int n = g.vGridN;
    auto blk = [&](double v, double lo, double hi) {
        return min(n - 1, max(0, static_cast<int>((v - lo) / ((hi - lo) / n))));
    };
    int c = g.vBlkRep[(blk(x, g.ext[0], g.ext[3]) * n + blk(y, g.ext[1], g.ext[4])) * n + blk(z, g.ext[2], g.ext[5])];
    for (int guard = 0; guard < 100000; ++guard)
    {
        const double* p = g.vSites + 3 * static_cast<size_t>(c);
        double best = (p[0] - x) * (p[0] - x) + (p[1] - y) * (p[1] - y) + (p[2] - z) * (p[2] - z);
        int next = -1;
        for (int e = g.vNbBegin[c]; e < g.vNbBegin[c + 1]; ++e)
        {
            int j = __ldg(g.vNb + e);
            if (j < 0) continue;
            const double* q = g.vSites + 3 * static_cast<size_t>(j);
            double d = (q[0] - x) * (q[0] - x) + (q[1] - y) * (q[1] - y) + (q[2] - z) * (q[2] - z);
            if (d < best)
            {
                best = d;
                next = j;
            }
        }
        if (next < 0) return c;
        c = next;
    }
    return c;
}

// ---------------------------------------------------------------------------------------------
// Voronoi mesh, production walker (VoronoiMeshSnapshot::MySegmentGenerator::next,
// VoronoiMeshSnapshot.cpp:1089-1222). Each cell is one contiguous record in 16-byte units:
//   [0] site x, y (FP64)   [1] site z (FP64), cell index, face count n
//   [2, 2 + n4)            per face the outward unit normal n and the distance d of the face's plane
//                          from the site (half the site distance, or the distance to a domain wall)
//   [2 + n4, 2 + n4 + n4/4) per face the neighbour's record offset (16-byte units), or the wall id
//                          -1..-6, or kPad
// with n4 = n rounded up to a multiple of 4 (padding faces have n = 0 and are never ahead). A
// crossing reads one record and takes the next cell's offset from it: no index arrays between
// cells. On entering a cell the FP64 position is rebased to FP32 coordinates l relative to the
// site; the exit through a face is s = (d - n . l) / (n . k). The two smallest exits are
// re-decided in FP64 from the exact sites when they lie within a near-tie tolerance (FP32 would
// misorder near-degenerate faces). The face just crossed is skipped (a ray cannot re-enter a convex
// cell), and a cell without a positive exit falls back to the reference's eps step and an FP64
// nearest-site search. A start in a known cell (a scattering event's interaction cell) needs no
// search; other starts walk greedily over the Delaunay neighbours from a site of the search block.
// ---------------------------------------------------------------------------------------------
#ifndef SKG_VORONOI32_MIN_BLOCKS
#define SKG_VORONOI32_MIN_BLOCKS 3
#endif
#ifndef SKG_VORONOI32_REFILL
#define SKG_VORONOI32_REFILL 8
#endif
struct VoronoiRec32 : GenBase
{
    using Acc = float;
    static constexpr int kMinBlocks = SKG_VORONOI32_MIN_BLOCKS;
    static constexpr int kRefillMin = SKG_VORONOI32_REFILL;  // waiting lanes before a warp takes new tasks
    // one traversal kernel: the Voronoi walk's register footprint leaves no room for two resident
    // kernels (4.62e6 packets/s unsplit against 4.41e6 split on the Voronoi galaxy)
    static constexpr bool kSplit = false;
    static constexpr int kNone = -99;     // no previous cell (the wall ids -1..-6 are taken)
    static constexpr int kPad = -100;     // padding face
    int rec, prev;                        // record offsets of the current and the previous cell
    float kxf, kyf, kzf;
    int hint;                             // the start cell when the caller knows it, else -1

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int h = -1)
    {
        startRay(x, y, z, ux, uy, uz);
        hint = h;
        rec = -1;
        prev = kNone;
        kxf = static_cast<float>(ux);
        kyf = static_cast<float>(uy);
        kzf = static_cast<float>(uz);
    }

    SKG_D static void site(const GridDev& g, int r, double& x, double& y, double& z)
    {
        const double* h = reinterpret_cast<const double*>(g.vRec + r);
        x = __ldg(h);
        y = __ldg(h + 1);
        z = __ldg(h + 2);
    }

    // FP64 exit distance from the current position through the face towards `to` (a record offset
    // or a wall id) of the cell with site p (0 when the face is not ahead)
    SKG_D double exit64(const GridDev& g, double px, double py, double pz, int to) const
    {
        if (to >= 0)
        {
            double qx, qy, qz;
            site(g, to, qx, qy, qz);
            double nx = qx - px, ny = qy - py, nz = qz - pz;
            double nk = nx * kx + ny * ky + nz * kz;
            if (!(nk > 0)) return 0.;
            return (nx * (0.5 * (qx + px) - rx) + ny * (0.5 * (qy + py) - ry) + nz * (0.5 * (qz + pz) - rz)) / nk;
        }
        switch (to)
        {
            case -1: return (g.ext[0] - rx) / kx;
            case -2: return (g.ext[3] - rx) / kx;
            case -3: return (g.ext[1] - ry) / ky;
            case -4: return (g.ext[4] - ry) / ky;
            case -5: return (g.ext[2] - rz) / kz;
            case -6: return (g.ext[5] - rz) / kz;
        }
        return 0.;
    }

    SKG_D bool locateRec(const GridDev& g, int cellHint)
    {
        int c = cellHint >= 0 ? cellHint : voronoiLocate(g, rx, ry, rz);
        rec = c >= 0 ? __ldg(g.vRecOff + c) : -1;
        prev = kNone;
        return rec >= 0;
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        if (state == GS_UNKNOWN)
        {
            if (!moveInside(g.ext, g.eps)) return false;
            if (!locateRec(g, (hint >= 0 && ds == 0.) ? hint : -1))
            {
                state = GS_OUTSIDE;
                return false;
            }
            if (ds > 0.) return true;
        }
        for (int guard = 0; guard < 64; ++guard)
        {
            const float4* R = g.vRec + rec;
            float4 h0 = __ldg(R), h1 = __ldg(R + 1);
            // the FP64 site only rebases the position here (the near-tie branch reloads it)
            float lx = static_cast<float>(rx - __hiloint2double(__float_as_int(h0.y), __float_as_int(h0.x)));
            float ly = static_cast<float>(ry - __hiloint2double(__float_as_int(h0.w), __float_as_int(h0.z)));
            float lz = static_cast<float>(rz - __hiloint2double(__float_as_int(h1.y), __float_as_int(h1.x)));
            int cell = __float_as_int(h1.z);
            int n4 = (__float_as_int(h1.w) + 3) & ~3;
            const float4* E = R + 2;
            const int4* ids = reinterpret_cast<const int4*>(R + 2 + n4);
            // the two nearest exits me / nk, compared by cross-multiplication so that only those two
            // distances take a division
            float meB = 0.f, nkB = 1.f, meS = 0.f, nkS = 1.f, scale = 0.f;
            int ib = kNone, is = kNone;
            for (int c = 0; c < n4; c += 4)
            {
                // four faces per step: their loads are issued together
                float4 q[4] = {__ldg(E + c), __ldg(E + c + 1), __ldg(E + c + 2), __ldg(E + c + 3)};
                int4 id4 = __ldg(ids + (c >> 2));
                int id[4] = {id4.x, id4.y, id4.z, id4.w};
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    float nk = q[j].x * kxf + q[j].y * kyf + q[j].z * kzf;
                    if (!(nk > 0.f) || id[j] == prev) continue;
                    float me = q[j].w - (q[j].x * lx + q[j].y * ly + q[j].z * lz);
                    if (!(me > 0.f)) continue;
                    if (ib == kNone || me * nkB < meB * nk)
                    {
                        meS = meB;
                        nkS = nkB;
                        is = ib;
                        meB = me;
                        nkB = nk;
                        ib = id[j];
                        scale = q[j].w;
                    }
                    else if (is == kNone || me * nkS < meS * nk)
                    {
                        meS = me;
                        nkS = nk;
                        is = id[j];
                    }
                }
            }
            if (ib == kNone)
            {
                // no exit ahead (the point sits on an edge or slightly outside the cell): the
                // reference's eps step and a fresh nearest-site search
                propagater(g.eps);
                if (!locateRec(g, -1))
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                continue;
            }
            const float best = meB / nkB, second = is != kNone ? meS / nkS : FLT_MAX;
            double sq = best;
            if (is != kNone && second - best <= 2e-5f * (best + scale))
            {
                // near tie: decide with the exact FP64 sites
                double px, py, pz;
                site(g, rec, px, py, pz);
                double s1 = exit64(g, px, py, pz, ib), s2 = exit64(g, px, py, pz, is);
                if (s2 > 0. && (s2 < s1 || !(s1 > 0.)))
                {
                    ib = is;
                    sq = s2;
                }
                else if (s1 > 0.)
                {
                    sq = s1;
                }
            }
            m = cell;
            ds = sq;
            propagater(sq);
            prev = rec;
            rec = ib;
            if (rec < 0) state = GS_OUTSIDE;
            return true;
        }
        state = GS_OUTSIDE;
        return false;
    }
};


// ---------------------------------------------------------------------------------------------
// Tetrahedral mesh, production walker (TetraMeshSpatialGrid::MySegmentGenerator::next,
// TetraMeshSpatialGrid.cpp:688-831). Every step reads one 128-byte record (TetRec) of the current
// tetrahedron: the exit is the nearest face plane ahead, s_f = (c_f - n_f . r) / (n_f . k) over the
// faces with n_f . k > 0 other than the face just entered (a ray cannot re-enter a convex cell),
// with the plane offset difference in FP64 and the division in FP32. Shared faces are one plane
// seen from both sides, so the walk stays watertight. The float planes are tilted from the exact
// ones by up to ~1e-7 of a tetrahedron's size; a decision within that bound of an edge, a vertex or
// a tie between two faces is re-taken in FP64 by the reference's Plucker decision (teLeavingFace),
// so that the cell sequence is the reference's.
// As the reference, the last in-mesh segment is dropped when the path leaves the hull. A start at a
// known cell (a scattering event's interaction cell) needs no point location; otherwise a walk over
// the face planes from the search block's representative finds the containing tetrahedron.
// ---------------------------------------------------------------------------------------------
// a record in registers (the fields are picked with selects, never by a dynamic index, so that the
// record stays out of local memory)
struct TetRegs
{
    double c[4];
    float n[12];
    int nb[4];
    int nface;

    SKG_D static TetRegs load(const TetRec* rec)
    {
        const float4* q = reinterpret_cast<const float4*>(rec);
        float4 a = __ldg(q), b = __ldg(q + 1), n0 = __ldg(q + 2), n1 = __ldg(q + 3), n2 = __ldg(q + 4), nb = __ldg(q + 5),
               nf = __ldg(q + 6);
        TetRegs t;
        t.c[0] = __hiloint2double(__float_as_int(a.y), __float_as_int(a.x));
        t.c[1] = __hiloint2double(__float_as_int(a.w), __float_as_int(a.z));
        t.c[2] = __hiloint2double(__float_as_int(b.y), __float_as_int(b.x));
        t.c[3] = __hiloint2double(__float_as_int(b.w), __float_as_int(b.z));
        t.n[0] = n0.x; t.n[1] = n0.y; t.n[2] = n0.z; t.n[3] = n0.w;
        t.n[4] = n1.x; t.n[5] = n1.y; t.n[6] = n1.z; t.n[7] = n1.w;
        t.n[8] = n2.x; t.n[9] = n2.y; t.n[10] = n2.z; t.n[11] = n2.w;
        t.nb[0] = __float_as_int(nb.x); t.nb[1] = __float_as_int(nb.y);
        t.nb[2] = __float_as_int(nb.z); t.nb[3] = __float_as_int(nb.w);
        t.nface = __float_as_int(nf.x);
        return t;
    }

    SKG_D int neighbour(int f) const { return f == 0 ? nb[0] : f == 1 ? nb[1] : f == 2 ? nb[2] : nb[3]; }

    // positive when (x, y, z) lies outside face F's plane
    template<int F>
    SKG_D double excess(double x, double y, double z) const
    {
        return static_cast<double>(n[3 * F]) * x + static_cast<double>(n[3 * F + 1]) * y + static_cast<double>(n[3 * F + 2]) * z - c[F];
    }
};

SKG_D int tetraLocate(const GridDev& g, double x, double y, double z)
{
    if (!GenBase::boxContains(g.ext, x, y, z)) return -1;
    const int n = g.teGridN;
    auto blk = [&](double v, double lo, double hi) {
        return min(n - 1, max(0, static_cast<int>(n * (v - lo) / (hi - lo))));
    };
    int t = g.teBlkRep[(blk(x, g.ext[0], g.ext[3]) * n + blk(y, g.ext[1], g.ext[4])) * n + blk(z, g.ext[2], g.ext[5])];
    // visibility walk: cross the face whose plane the point is farthest outside of
    for (int guard = 0; guard < 4096 && t >= 0; ++guard)
    {
        TetRegs r = TetRegs::load(g.teRec + t);
        int f = -1;
        double worst = 0., e;
        if ((e = r.excess<0>(x, y, z)) > worst) { worst = e; f = 0; }
        if ((e = r.excess<1>(x, y, z)) > worst) { worst = e; f = 1; }
        if ((e = r.excess<2>(x, y, z)) > worst) { worst = e; f = 2; }
        if ((e = r.excess<3>(x, y, z)) > worst) { worst = e; f = 3; }
        if (f < 0) return t;
        t = r.neighbour(f);
    }
    return tetraCellIndex(g, x, y, z);  // walk left the hull or did not settle: the reference's block scan
}

#ifndef SKG_TETRA32_MIN_BLOCKS
#define SKG_TETRA32_MIN_BLOCKS 3
#endif
struct TetraPlane32 : GenBase
{
    using Acc = float;
    static constexpr int kMinBlocks = SKG_TETRA32_MIN_BLOCKS;
    static constexpr int kRefillMin = 8;  // waiting lanes before a warp takes new tasks
    // bound on the displacement of a float plane from its exact one, in units of eps (1e-12 of the
    // domain diagonal): 2^-24 per normal component over at most the diagonal, with margin
    static constexpr double kTilt = 1.6e5;
    static constexpr float kNk = 1e-6f;  // |n.k| below this may have either sign in exact arithmetic
    int mr, ef;  // current tetrahedron, face it was entered through (-1: none)
    int hint;
    float kxf, kyf, kzf;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int h = -1)
    {
        startRay(x, y, z, ux, uy, uz);
        hint = h;
        mr = -1;
        ef = -1;
        kxf = static_cast<float>(ux);
        kyf = static_cast<float>(uy);
        kzf = static_cast<float>(uz);
    }

    // whether the float exit decision in tetrahedron r may differ from the exact one: the point lies
    // within tol of the exit plane, the two nearest exits lie within the planes' error of each other
    // (an edge or a vertex), or a face almost parallel to the path lies within tol of the point
    SKG_D bool ambiguous(const TetRegs& r, double x, double y, double z, float tol) const
    {
        float best = FLT_MAX, second = FLT_MAX, nkBest = 1.f, nkSecond = 1.f;
        float inside = FLT_MAX, graze = FLT_MAX;
        auto face = [&](auto F) {
            constexpr int f = decltype(F)::value;
            if (f == ef) return;
            float nk = r.n[3 * f] * kxf + r.n[3 * f + 1] * kyf + r.n[3 * f + 2] * kzf;
            float me = static_cast<float>(-r.template excess<f>(x, y, z));
            if (!(nk > 0.f))
            {
                if (nk > -kNk) graze = fminf(graze, me);  // may be a face ahead in exact arithmetic
                return;
            }
            float s = me / nk;
            if (s < best)
            {
                second = best;
                nkSecond = nkBest;
                best = s;
                nkBest = nk;
                inside = me;
            }
            else if (s < second)
            {
                second = s;
                nkSecond = nk;
            }
        };
        face(std::integral_constant<int, 0>());
        face(std::integral_constant<int, 1>());
        face(std::integral_constant<int, 2>());
        face(std::integral_constant<int, 3>());
        // second - best < tol (1/nkBest + 1/nkSecond) + 1e-6 second, multiplied through by the
        // positive nkBest nkSecond (the bound is far coarser than the rounding of the test)
        return inside < tol || graze < tol + 1e-6f * best ||
               (second < FLT_MAX &&
                (second - best) * nkBest * nkSecond < tol * (nkBest + nkSecond) + 1e-6f * second * nkBest * nkSecond);
    }

    SKG_D bool next(const GridDev& g)
    {
        if (state == GS_OUTSIDE) return false;
        if (state == GS_UNKNOWN)
        {
            if (!moveInside(g.ext, g.eps)) return false;
            mr = (hint >= 0 && ds == 0.) ? hint : tetraLocate(g, rx, ry, rz);
            ef = -1;
            if (mr < 0)
            {
                state = GS_OUTSIDE;
                return false;
            }
            if (ds > 0.) return true;
        }
        // the float planes (normals rounded to FP32, offsets through a shared vertex, so neighbours
        // agree) lie within kTilt * eps = 1.6e-7 of the domain diagonal of the exact ones
        const float tol = static_cast<float>(kTilt * g.eps);
        for (int guard = 0; guard < 256; ++guard)
        {
            TetRegs r = TetRegs::load(g.teRec + mr);
            // the nearest exit me / nk over the faces ahead (nk > 0), compared by cross-multiplication
            // so that only the chosen face's distance takes a division
            float meBest = 0.f, nkBest = 1.f;
            int lf = -1;
            auto face = [&](auto F) {
                constexpr int f = decltype(F)::value;
                float nk = r.n[3 * f] * kxf + r.n[3 * f + 1] * kyf + r.n[3 * f + 2] * kzf;
                if (f == ef || !(nk > 0.f)) return;
                float me = static_cast<float>(-r.template excess<f>(rx, ry, rz));
                if (lf < 0 || me * nkBest < meBest * nk)
                {
                    meBest = me;
                    nkBest = nk;
                    lf = f;
                }
            };
            face(std::integral_constant<int, 0>());
            face(std::integral_constant<int, 1>());
            face(std::integral_constant<int, 2>());
            face(std::integral_constant<int, 3>());
            const float best = lf >= 0 ? meBest / nkBest : FLT_MAX;
            // Between two interior faces either choice continues the walk from the same point; only
            // in a tetrahedron on the hull can a float decision end the path where the reference's
            // goes on (or the reverse), so only there is the decision tested, in a second pass.
            if (lf >= 0 && ((r.nb[0] | r.nb[1] | r.nb[2] | r.nb[3]) >= 0 || !ambiguous(r, rx, ry, rz, tol)))
            {
                int nt = r.neighbour(lf);
                int nf = (r.nface >> (8 * lf)) & 0xff;
                if (best > 0.f)
                {
                    m = mr;
                    ds = best;
                    propagater(ds);
                }
                mr = nt;
                ef = nf;
                if (mr < 0)
                {
                    // the reference drops the final in-mesh segment when the path leaves the hull
                    state = GS_OUTSIDE;
                    return false;
                }
                if (best > 0.f) return true;
                continue;
            }
            // no face ahead, or a decision within the float planes' error of an edge, a vertex or a
            // tie: re-taken in FP64 the reference's way
            double d;
            int xf = teLeavingFace(g, mr, ef, rx, ry, rz, kx, ky, kz, d);
            if (xf == -1 || d < g.eps)
            {
                // no exit point: the reference's eps step and its own point location
                propagater(g.eps);
                mr = tetraCellIndex(g, rx, ry, rz);
                ef = -1;
                if (mr < 0)
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                continue;
            }
            m = mr;
            ds = d;
            propagater(d);
            ef = g.teNFace[4 * static_cast<size_t>(mr) + xf];
            mr = g.teNTet[4 * static_cast<size_t>(mr) + xf];
            if (mr < 0)
            {
                state = GS_OUTSIDE;
                return false;
            }
            return true;
        }
        state = GS_OUTSIDE;
        return false;
    }
};

// ---------------------------------------------------------------------------------------------
// 1D spherical grid, production: the reference-order FP64 shell crossings (a handful of square
// roots per ray over a border table that stays in L1) with FP32 accumulators like the other
// production walkers.
// ---------------------------------------------------------------------------------------------
struct Sphere1DFast : Sphere1DExact
{
    using Acc = float;
};

// 2D cylindrical grid, production: the reference-order FP64 crossings with FP32 accumulators
struct Cylinder2DFast : Cylinder2DExact
{
    using Acc = float;
};

// 2D spherical grid, production: the reference-order FP64 crossings with FP32 accumulators
struct Sphere2DFast : Sphere2DExact
{
    using Acc = float;
};

// 3D spherical grid, production: the reference-order FP64 crossings with FP32 accumulators
struct Sphere3DFast : Sphere3DExact
{
    using Acc = float;
};

// 3D cylindrical grid, production: the reference-order FP64 crossings with FP32 accumulators
struct Cylinder3DFast : Cylinder3DExact
{
    using Acc = float;
};

}  // namespace skg
