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
    int i, j, k;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz)
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

template<typename Real>
struct OctreeFast : FastBase<Real>
{
    int node;

    SKG_D void start(const GridDev&, double x, double y, double z, double ux, double uy, double uz)
    {
        this->startFast(x, y, z, ux, uy, uz);
        node = -1;
    }

    SKG_D bool next(const GridDev& g)
    {
        if (this->state == GS_OUTSIDE) return false;
        if (this->state == GS_UNKNOWN)
        {
            if (!this->moveInside(g.ext, g.eps)) return false;
            node = octreeLeafChild(g, this->rx, this->ry, this->rz);
            if (node < 0)
            {
                this->state = GS_OUTSIDE;
                return false;
            }
            if (this->ds > 0.) return true;
        }
        const double* b = g.tBounds + 6 * static_cast<size_t>(node);
        int sx = this->kx < 0.0 ? 0 : 3, sy = this->ky < 0.0 ? 1 : 4, sz = this->kz < 0.0 ? 2 : 5;
        double xE = b[sx], yE = b[sy], zE = b[sz];
        Real d;
        int a = this->pickAxis(this->dist(xE, this->rx, this->ikx, this->kx), this->dist(yE, this->ry, this->iky, this->ky),
                               this->dist(zE, this->rz, this->ikz, this->kz), false, d);
        int wall = 2 * a + ((a == 0 ? this->kx : (a == 1 ? this->ky : this->kz)) < 0.0 ? 0 : 1);
        this->m = g.tCell[node];
        this->ds = d;
        this->rebase(a, a == 0 ? xE : (a == 1 ? yE : zE), this->ds);
        // first neighbour across the wall whose face contains the exit point (TreeNode::neighbor);
        // the normal coordinate lies on the wall, so only the transverse ranges are tested
        int nb = -1;
        int e0 = g.tNbBegin[6 * node + wall], e1 = g.tNbBegin[6 * node + wall + 1];
        for (int e = e0; e < e1; ++e)
        {
            int cand = g.tNb[e];
            const double* c = g.tBounds + 6 * static_cast<size_t>(cand);
            bool in = (a == 0 || (this->rx >= c[0] && this->rx <= c[3])) && (a == 1 || (this->ry >= c[1] && this->ry <= c[4]))
                      && (a == 2 || (this->rz >= c[2] && this->rz <= c[5]));
            if (in)
            {
                nb = cand;
                break;
            }
        }
        if (nb < 0)
        {
            // no neighbour (domain wall, or a corner exit): locate the point just beyond the wall
            double e = g.eps;
            nb = octreeLeafChild(g, this->rx + this->kx * e, this->ry + this->ky * e, this->rz + this->kz * e);
        }
        if (nb == node)
        {
            // still in the same node: escape to the next representable coordinates (as the reference)
            this->rx = nextafter(this->rx, (this->kx < 0.) ? -DBL_MAX : DBL_MAX);
            this->ry = nextafter(this->ry, (this->ky < 0.) ? -DBL_MAX : DBL_MAX);
            this->rz = nextafter(this->rz, (this->kz < 0.) ? -DBL_MAX : DBL_MAX);
            nb = octreeLeafChild(g, this->rx, this->ry, this->rz);
        }
        if (nb < 0 || nb == node) this->state = GS_OUTSIDE;
        node = nb;
        return true;
    }
};

}  // namespace skg
