// Production walkers: the reference generators' geometry with FP32 distance arithmetic.
//
// Each walker keeps the entry point of the current cell in FP64 and re-bases it at every crossing
// (the coordinate of the crossed wall is set exactly, the others advance along the ray), so that all
// per-cell geometry is computed in FP32 relative to that point: wall offsets (FP64 difference,
// rounded once to FP32) times the precomputed FP32 inverse direction. There are no divisions per
// crossing and the exit-axis selection is branch free. Exit-axis ties follow the reference's rule.
// Errors against the FP64 walkers are a few FP32 ulps of the cell size per segment; cell sequences
// differ only where a ray passes within that distance of a cell edge or corner.
#pragma once

#include <type_traits>

#include "grids.cuh"

namespace skg {

template<typename Real>
struct RealLimits;
template<>
struct RealLimits<float>
{
    SKG_D static float big() { return FLT_MAX; }
};
template<>
struct RealLimits<double>
{
    SKG_D static double big() { return DBL_MAX; }
};

// common part: exact moveInside (once per ray, FP64, as the reference) and the inverse direction
template<typename Real>
struct FastBase : GenBase
{
    Real ikx, iky, ikz;

    SKG_D void startFast(double x, double y, double z, double ux, double uy, double uz)
    {
        startRay(x, y, z, ux, uy, uz);
        const Real big = RealLimits<Real>::big();
        ikx = fabs(ux) > 1e-15 ? Real(1) / Real(ux) : big;
        iky = fabs(uy) > 1e-15 ? Real(1) / Real(uy) : big;
        ikz = fabs(uz) > 1e-15 ? Real(1) / Real(uz) : big;
    }

    // distance from the entry point to the wall at coordinate w along an axis (FP32 after one FP64 difference)
    SKG_D static Real dist(double w, double r, Real ik, double k)
    {
        return fabs(k) > 1e-15 ? Real(w - r) * ik : RealLimits<Real>::big();
    }

    // selects the exit axis with the reference's tie rule (x if dx<=dy && dx<=dz, y if dy<dx && dy<=dz
    // for the Cartesian grid; the octree uses dy<=dx) and rebases the entry point on the exit wall
    SKG_D int pickAxis(Real dx, Real dy, Real dz, bool yStrict, Real& d) const
    {
        bool isx = dx <= dy && dx <= dz;
        bool isy = !isx && (yStrict ? dy < dx : dy <= dx) && dy <= dz;
        int a = isx ? 0 : (isy ? 1 : 2);
        d = isx ? dx : (isy ? dy : dz);
        return a;
    }

    SKG_D void rebase(int axis, double wall, double d)
    {
        double nx = rx + kx * d, ny = ry + ky * d, nz = rz + kz * d;
        rx = axis == 0 ? wall : nx;
        ry = axis == 1 ? wall : ny;
        rz = axis == 2 ? wall : nz;
    }
};

template<typename Real>
struct CartesianFast : FastBase<Real>
{
    using Acc = Real;
    static constexpr int kMinBlocks = 4;
    static constexpr int kRefillMin = 16;  // waiting lanes before a warp takes new tasks
    int i, j, k;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int = -1)
    {
        this->startFast(x, y, z, ux, uy, uz);
    }

    SKG_D bool next(const GridDev& g)
    {
        if (this->state == GS_OUTSIDE) return false;
        if (this->state == GS_UNKNOWN)
        {
            if (!this->moveInside(g.ext, xmul(1e-12, boxDiagonal(g.ext)))) return false;
            i = locateClip(g.xb, g.nx + 1, this->rx);
            j = locateClip(g.yb, g.ny + 1, this->ry);
            k = locateClip(g.zb, g.nz + 1, this->rz);
            if (this->ds > 0.) return true;
        }
        int sx = this->kx < 0.0 ? 0 : 1, sy = this->ky < 0.0 ? 0 : 1, sz = this->kz < 0.0 ? 0 : 1;
        double xE = g.xb[i + sx], yE = g.yb[j + sy], zE = g.zb[k + sz];
        Real d;
        int a = this->pickAxis(this->dist(xE, this->rx, this->ikx, this->kx), this->dist(yE, this->ry, this->iky, this->ky),
                               this->dist(zE, this->rz, this->ikz, this->kz), true, d);
        this->m = k + g.nz * j + g.nz * g.ny * i;
        this->ds = d;
        this->rebase(a, a == 0 ? xE : (a == 1 ? yE : zE), this->ds);
        i += a == 0 ? 2 * sx - 1 : 0;
        j += a == 1 ? 2 * sy - 1 : 0;
        k += a == 2 ? 2 * sz - 1 : 0;
        if (i < 0 || i >= g.nx || j < 0 || j >= g.ny || k < 0 || k >= g.nz) this->state = GS_OUTSIDE;
        return true;
    }
};

// Octree walker on the leaf-indexed FP32 records. The current cell's record (bounds, density,
// neighbour-list base) and wall counts are held in registers; a crossing loads the ids of the exit
// wall's neighbours and their records until one contains the exit point, and that record becomes
// the current one (two dependent loads per crossing, all from a working set that stays in L2).
// resident 256-thread blocks per SM requested for the FP32 octree trace kernel (register limit)
#ifndef SKG_OCTREE32_MIN_BLOCKS
#define SKG_OCTREE32_MIN_BLOCKS 4
#endif

struct OctreeLeaf32 : FastBase<float>
{
    using Acc = float;
    static constexpr int kMinBlocks = SKG_OCTREE32_MIN_BLOCKS;
    static constexpr int kRefillMin = 16;  // waiting lanes before a warp takes new tasks
    int cell;
    float4 ra, rb;                 // bounds, density and list base of the current cell (record words 0-1)
    float segDens;                 // density of the cell of the segment just returned
    int hint;                      // the start cell when the caller knows it (an interaction cell), else -1

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz, int h = -1)
    {
        this->startFast(x, y, z, ux, uy, uz);
        cell = -1;
        hint = h;
    }

    SKG_D double density(const double*) const { return static_cast<double>(segDens); }

    SKG_D void enter(const GridDev& g, int c)
    {
        cell = c;
        ra = __ldg(g.tLeaf + 4 * static_cast<size_t>(c));
        rb = __ldg(g.tLeaf + 4 * static_cast<size_t>(c) + 1);
    }

    // top-down location of the leaf containing a point (FP64 bounds), as a cell index
    SKG_D static int locate(const GridDev& g, double x, double y, double z)
    {
        int n = octreeLeafChild(g, x, y, z);
        return n < 0 ? -1 : g.tCell[n];
    }

    // half-open interval test in the direction of travel: a point on the boundary belongs to the
    // interval the ray moves into (closed on both ends for a zero direction component)
    SKG_D static bool within(float p, float lo, float hi, double k)
    {
        return k > 0.0 ? (p >= lo && p < hi) : (k < 0.0 ? (p > lo && p <= hi) : (p >= lo && p <= hi));
    }

    SKG_D bool next(const GridDev& g)
    {
        if (this->state == GS_OUTSIDE) return false;
        if (this->state == GS_UNKNOWN)
        {
            if (!this->moveInside(g.ext, g.eps)) return false;
            // a start inside the domain in a known cell needs no top-down search
            int c = (hint >= 0 && this->ds == 0.) ? hint : locate(g, this->rx, this->ry, this->rz);
            if (c < 0)
            {
                this->state = GS_OUTSIDE;
                return false;
            }
            enter(g, c);
            if (this->ds > 0.) return true;
        }
        double xE = this->kx < 0.0 ? ra.x : ra.w;
        double yE = this->ky < 0.0 ? ra.y : rb.x;
        double zE = this->kz < 0.0 ? ra.z : rb.y;
        float d;
        int a = this->pickAxis(this->dist(xE, this->rx, this->ikx, this->kx), this->dist(yE, this->ry, this->iky, this->ky),
                               this->dist(zE, this->rz, this->ikz, this->kz), false, d);
        // the entry point may lie a rounding error beyond a wall of a cell entered through the
        // fallback below: never step backwards, so that the walk advances monotonically
        d = fmaxf(d, 0.f);
        int wall = 2 * a + ((a == 0 ? this->kx : (a == 1 ? this->ky : this->kz)) < 0.0 ? 0 : 1);
        this->m = cell;
        this->ds = d;
        segDens = rb.z;
        this->rebase(a, a == 0 ? xE : (a == 1 ? yE : zE), this->ds);
        // words 2-3 of the record (same cache line as words 0-1): the list offsets and, per wall,
        // the single neighbour across it (-1: domain wall, -2: several neighbours)
        const int* w23 = reinterpret_cast<const int*>(g.tLeaf + 4 * static_cast<size_t>(cell) + 2);
        int one = __ldg(w23 + 2 + wall);
        int old = cell, nb = -1;
        if (one >= 0)
        {
            enter(g, one);
            return true;
        }
        if (one == -1)
        {
            this->state = GS_OUTSIDE;
            return true;
        }
        unsigned long long cnt = (static_cast<unsigned long long>(static_cast<unsigned>(__ldg(w23 + 1))) << 32)
                                 | static_cast<unsigned>(__ldg(w23));
        int base = __float_as_int(rb.w);
        bool listed = cnt != ~0ULL;
        int e0 = base + static_cast<int>((cnt >> (9 * wall)) & 511);
        int n = listed ? base + static_cast<int>((cnt >> (9 * (wall + 1))) & 511) - e0 : 0;
        float pu = static_cast<float>(a == 0 ? this->ry : this->rx);
        float pv = static_cast<float>(a == 2 ? this->ry : this->rz);
        double ku = a == 0 ? this->ky : this->kx;
        double kv = a == 2 ? this->ky : this->kz;
        for (int e = 0; e < n; ++e)
        {
            int c = __ldg(g.tLeafNb + e0 + e);
            float4 qa = __ldg(g.tLeaf + 4 * static_cast<size_t>(c)), qb = __ldg(g.tLeaf + 4 * static_cast<size_t>(c) + 1);
            float ulo = a == 0 ? qa.y : qa.x, uhi = a == 0 ? qb.x : qa.w;
            float vlo = a == 2 ? qa.y : qa.z, vhi = a == 2 ? qb.x : qb.y;
            if (within(pu, ulo, uhi, ku) && within(pv, vlo, vhi, kv))
            {
                nb = c;
                cell = c;
                ra = qa;
                rb = qb;
                break;
            }
        }
        if (nb < 0)
        {
            // No listed neighbour holds the exit point (a wall without list, or an exit point on a
            // cell edge). Move the point forward along every axis by a few FP32 roundings of the
            // coordinates (so that it lies beyond any FP32-rounded wall it sits on) and locate it
            // top-down in the FP64 tree; a point outside the domain ends the path.
            double big = fmax(fabs(this->rx), fmax(fabs(this->ry), fabs(this->rz)));
            double e = fmax(g.eps, 4.8e-7 * big);
            this->rx += this->kx > 0.0 ? e : (this->kx < 0.0 ? -e : 0.0);
            this->ry += this->ky > 0.0 ? e : (this->ky < 0.0 ? -e : 0.0);
            this->rz += this->kz > 0.0 ? e : (this->kz < 0.0 ? -e : 0.0);
            nb = locate(g, this->rx, this->ry, this->rz);
            if (nb >= 0 && nb != old) enter(g, nb);
        }
        if (nb < 0 || nb == old) this->state = GS_OUTSIDE;
        return true;
    }
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
            float best = FLT_MAX, second = FLT_MAX, scale = 0.f;
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
                    float s = (q[j].w - (q[j].x * lx + q[j].y * ly + q[j].z * lz)) / nk;
                    if (!(s > 0.f)) continue;
                    if (s < best)
                    {
                        second = best;
                        is = ib;
                        best = s;
                        ib = id[j];
                        scale = q[j].w;
                    }
                    else if (s < second)
                    {
                        second = s;
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
// seen from both sides, so the walk stays watertight: a point that rounding puts just past the exit
// plane gives a zero-length step into the neighbour, which is taken without reporting a segment.
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
        for (int guard = 0; guard < 256; ++guard)
        {
            TetRegs r = TetRegs::load(g.teRec + mr);
            float best = FLT_MAX;
            int lf = -1;
            auto face = [&](auto F) {
                constexpr int f = decltype(F)::value;
                float nk = r.n[3 * f] * kxf + r.n[3 * f + 1] * kyf + r.n[3 * f + 2] * kzf;
                if (f == ef || !(nk > 0.f)) return;
                float s = static_cast<float>(-r.template excess<f>(rx, ry, rz)) / nk;
                if (s < best)
                {
                    best = s;
                    lf = f;
                }
            };
            face(std::integral_constant<int, 0>());
            face(std::integral_constant<int, 1>());
            face(std::integral_constant<int, 2>());
            face(std::integral_constant<int, 3>());
            if (lf < 0)
            {
                // no face ahead (degenerate direction or position): the reference's eps step and a
                // fresh point location
                propagater(g.eps);
                mr = tetraLocate(g, rx, ry, rz);
                ef = -1;
                if (mr < 0)
                {
                    state = GS_OUTSIDE;
                    return false;
                }
                continue;
            }
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
