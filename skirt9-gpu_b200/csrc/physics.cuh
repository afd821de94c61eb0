// Device physics shared by the life-cycle stages: scene records, source launch, instrument
// projection, wavelength bins, warp-aggregated FP64 atomics.
#pragma once

#include "grids.cuh"
#include "guide.cuh"

namespace skg {

constexpr int MAX_INSTR = 16;
// distinct (instrument, wavelength bin, pixel) keys buffered per packet slot for the per-history
// statistics: with the wavefront's own buffers, and within the static scratch of the no-allocation run
constexpr int STATS_CAP = 128;
constexpr int STATS_CAP_NOALLOC = 48;
constexpr int MAX_SCATT_EVENTS = 1 << 20;

struct SourceDev
{
    int posModel, specModel;
    double pos[3];
    double geom[6];
    unsigned long long first, num;
    double Lpk;
    double xi, bmin, bmax;
    int toff, tsize, roff, rsize;
};

struct InstrDev
{
    int kind, same, stats, comps;
    int npx, npy, nbins, woff, wnb;
    double kobs[3];
    double ct, st, cp, sp, co, so;
    double xpmin, xpsiz, ypmin, ypsiz;
    double* ifu;        // frame total, nbins*npix, index l + ell*npix
    double* sed;        // SED total, nbins
    double* ifuComp;    // 3 planes: transparent, direct, scattered
    double* sedComp;
    double* ifuStats;   // 5 planes: sum w^k, k = 0..4
    double* sedStats;
    int levels;             // scattering-level planes after the 3 component planes (primary packets)
    int nband;              // > 0: band wavelength grid of nband bands in place of the disjoint grid
    const int* bandBeg;     // nband + 1 offsets into the band tables
    const double* bandLam;  // band tables: increasing wavelengths
    const double* bandTr;   // normalised transmissions
    const double* bandW;    // nband effective widths
    double zfac;            // 1 + observer-frame redshift
    double apR2;            // SED aperture radius squared (0: no aperture)
};

// The prepared secondary (dust) emission source of a segment (DustSecondarySource with the
// AllCellsLibrary: launch order = cell order). Histories [Iv[m], Iv[m+1]) launch from cell m.
struct SecondaryDev
{
    const unsigned long long* Iv;  // numCells + 1 first history index per cell
    const double* Lv;              // numCells normalised cell luminosities
    const double* Wv;              // numCells composite-biased launch weights
    const double* xv;              // npts wavelengths of the emission spectra (NR::cdf axis)
    const double* pv;              // numCells * npts normalised emission pdf per cell
    const double* Pv;              // numCells * npts normalised emission cdf per cell
    const int* cellNode;           // octree: leaf node of each cell (its extent is the cell box)
    int npts, numCells;
    double Lpk;                    // _Lpp * Lv_s / Wv_s of SecondarySourceSystem (one source)
    double xi;                     // DustEmissionOptions::wavelengthBias
    double logMin, logWidth, bmin, bmax;  // its LogWavelengthDistribution
};

// read-only scene data of a run
struct alignas(16) Scene  // 16-byte multiple: a batch stages its scene table as int4 words
{
    GridDev g;
    const double* dens;
    const double* mixLb;
    const double* mixExt;
    const double* mixSca;
    const double* mixG;
    int nmix;

    int nsrc;
    const SourceDev* src;
    const double* tabL;
    const double* tabA;
    const double* tabB;
    const double* radR;
    const double* radP;

    int ninstr;
    const InstrDev* instr;
    const double* wlgB;
    const int* wlgEll;

    int rfOn, nrf, rfNb;
    const double* rfB;
    const int* rfEll;
    double* rf;

    int forced, minScatt, peel;
    int explicitAbs;  // explicit absorption: sampling on scattering optical depth, weight exp(-tau_abs)
    double minWeightRed, pathLengthBias;
    unsigned long long seed;

    // learned path guiding: 0 off, 1 pilot (record scattering events), 2 guided scattering
    int guideMode;
    int guideTarget;                 // instrument whose detections define the records' importance
    float guideAlpha;                // probability of sampling the network's lobes (mode 2)
    float guideRecFrac;              // fraction of scattering events recorded (mode 1)
    GuideRecord* guideRec;
    unsigned long long* guideRecCount;
    unsigned long long guideRecCap;
    const float* guideImportance;    // per-pixel weight of the target frame's detections (null: 1)
    const unsigned char* guideBlob;  // packed BF16 network (mode 2)
    int* guideErr;
    // secondary-emission segment: the prepared dust source (null for primary emission)
    const SecondaryDev* sec;
};

// atomicAdd after summing the contributions of the warp's active lanes that target the same address
SKG_D void atomicAddAgg(double* addr, double v)
{
    unsigned active = __activemask();
    unsigned peers = __match_any_sync(active, reinterpret_cast<unsigned long long>(addr));
    int leader = __ffs(peers) - 1;
    double sum = 0.;
    unsigned rem = peers;
    while (rem)
    {
        int j = __ffs(rem) - 1;
        rem &= rem - 1;
        sum += __shfl_sync(peers, v, j);
    }
    if ((threadIdx.x & 31) == leader) atomicAdd(addr, sum);
}

// DisjointWavelengthGrid::bin (DisjointWavelengthGrid.cpp:333-342)
SKG_D int wlgBin(const double* borders, int nb, const int* ellv, double lambda)
{
    return ellv[upperBound(borders, nb, lambda)];
}

// Band::transmission (SKIRT/core/Band.cpp): NR::interpolateLinLin in the normalised transmission
// table (zero outside it), scaled to relative transmission by the effective width
SKG_D double bandTransmission(const double* lv, const double* tv, int size, double width, double lambda)
{
    int index = upperBound(lv, size, lambda);
    if (index == 0 || index >= size) return 0.;
    double T = tv[index - 1] + ((lambda - lv[index - 1]) / (lv[index] - lv[index - 1])) * (tv[index] - tv[index - 1]);
    return T * width;
}

// SpecialFunctions::gexp(p, x) (SKIRT/utils/SpecialFunctions.cpp:822-836), the inverse of the
// generalized logarithm used by Random::cdfLogLog (Random.cpp:200-207)
SKG_D double gexp(double p, double x)
{
    const double q = 1.0 - p;
    if (q == 0.0) return exp(x);
    if (fabs(q) < 1e-3)
    {
        double x2 = x * x;
        return exp(x)
               * (1.0 - 0.5 * x2 * q + 1.0 / 24.0 * x * x2 * (8.0 + 3.0 * x) * q * q
                  - 1.0 / 48.0 * x2 * x2 * (12.0 + 8.0 * x + x2) * q * q * q);
    }
    return pow(1.0 + q * x, 1.0 / q);
}

// Lambert W, branch -1, for x in [-1/e, 0): Halley iteration (Corless et al. 1996) from the
// branch-point series or the asymptotic expansion
SKG_D double lambertWm1(double x)
{
    if (x >= 0.) return -INFINITY;
    if (x <= -1. / M_E) return -1.;
    double w;
    if (x < -0.25)
    {
        double pp = -sqrt(2. * (M_E * x + 1.));
        w = -1. + pp - pp * pp / 3. + 11. / 72. * pp * pp * pp;
    }
    else
    {
        double l1 = log(-x), l2 = log(-l1);
        w = l1 - l2 + l2 / l1;
    }
    for (int it = 0; it < 20; ++it)
    {
        double ew = exp(w);
        double f = w * ew - x;
        double wp1 = w + 1.;
        if (wp1 == 0.) break;
        double dw = f / (ew * wp1 - (w + 2.) * f / (2. * wp1));
        w -= dw;
        if (fabs(dw) <= 1e-15 * fabs(w)) break;
    }
    return w;
}

// launched packet state
struct Launched
{
    double x, y, z, kx, ky, kz, L, lambda;
};

// SecondarySourceSystem::launch -> DustSecondarySource::launch / launchFromCell
// (SecondarySourceSystem.cpp:118-133, DustSecondarySource.cpp:521-626): the cell from the history
// index, the wavelength from the cell's emission spectrum (Random::cdfLogLog) or the log-uniform
// bias distribution with its compensating weight (NR::value<NR::interpolateLogLog>), a uniform
// position in the cell box (Random::position, Box::fracPos), an isotropic direction
SKG_D Launched launchSecondary(const Scene& p, unsigned long long hist, Rng& rng)
{
    const SecondaryDev& S = *p.sec;
    int m = upperBound(S.Iv, S.numCells + 1, hist) - 1;
    m = min(max(m, 0), S.numCells - 1);
    double ws = S.Lv[m] / S.Wv[m];
    const double* xv = S.xv;
    const double* pv = S.pv + static_cast<size_t>(m) * S.npts;
    const double* Pv = S.Pv + static_cast<size_t>(m) * S.npts;
    const int n = S.npts;
    auto fromSpectrum = [&]() {
        double X = rng.uniform();
        int i = locateClip(Pv, n, X);
        double alpha = log(pv[i + 1] / pv[i]) / log(xv[i + 1] / xv[i]);
        return xv[i] * gexp(-alpha, (X - Pv[i]) / (pv[i] * xv[i]));
    };
    double lambda, w;
    if (!S.xi)
    {
        lambda = fromSpectrum();
        w = 1.;
    }
    else
    {
        if (rng.uniform() > S.xi)
            lambda = fromSpectrum();
        else
            lambda = exp(S.logMin + S.logWidth * rng.uniform());
        // NR::value<NR::interpolateLogLog>: 0 outside the spectrum's grid
        double s = 0.;
        if (!(lambda > xv[n - 1]))
        {
            int jl = -1, ju = n - 1;
            while (ju - jl > 1)
            {
                int jm = (ju + jl) >> 1;
                if (lambda < xv[jm]) ju = jm; else jl = jm;
            }
            if (jl >= 0) s = interpLogLog(lambda, xv[jl], xv[jl + 1], pv[jl], pv[jl + 1]);
        }
        if (!s)
            w = 0.;
        else
        {
            // LogWavelengthDistribution::probability, Range::containsFuzzy (relative 1e-14)
            double b = (lambda >= S.bmin * (1 - 1e-14) && lambda <= S.bmax * (1 + 1e-14)) ? 1. / (S.logWidth * lambda) : 0.;
            w = s / ((1 - S.xi) * s + S.xi * b);
        }
    }
    // a random position in cell m (SpatialGrid::randomPositionInCell of the grid kind)
    Launched o;
    if (p.g.kind == 3)
    {
        // TetraMeshSpatialGrid::Tetra::generatePosition / generateBarycentric
        // (TetraMeshSpatialGrid.cpp:140-173): the unit cube folded into the tetrahedron
        double s = rng.uniform(), t = rng.uniform(), u = rng.uniform();
        if (xadd(s, t) > 1.)
        {
            s = xsub(1., s);
            t = xsub(1., t);
        }
        if (xadd(t, u) > 1.)
        {
            double tmp = u;
            u = xsub(xsub(1., s), t);
            t = xsub(1., tmp);
        }
        else if (xadd(xadd(s, t), u) > 1.)
        {
            double tmp = u;
            u = xsub(xadd(xadd(s, t), u), 1.);
            s = xsub(xsub(1., t), tmp);
        }
        double r = xsub(xsub(xsub(1., u), t), s);
        double v[4][3];
        for (int q = 0; q < 4; ++q) teVertex(p.g, m, q, v[q][0], v[q][1], v[q][2]);
        double c[3];
        for (int a = 0; a < 3; ++a)
            c[a] = xadd(xadd(xadd(xmul(r, v[0][a]), xmul(u, v[1][a])), xmul(t, v[2][a])), xmul(s, v[3][a]));
        o.x = c[0];
        o.y = c[1];
        o.z = c[2];
    }
    else if (p.g.kind == 4)
    {
        // Sphere1DSpatialGrid::randomPositionInCell (Sphere1DSpatialGrid.cpp:80-91): an isotropic
        // direction, then r^3 uniform between the shell's borders (Cubic::pow3)
        double ux, uy, uz;
        isotropicDirection(rng, ux, uy, uz);
        double r0 = p.g.sRv[m], r1 = p.g.sRv[m + 1];
        double d3 = xmul(xsub(r1, r0), xadd(xadd(xmul(r1, r1), xmul(r1, r0)), xmul(r0, r0)));
        double r = cbrt(xadd(xmul(xmul(r0, r0), r0), xmul(d3, rng.uniform())));
        o.x = xmul(r, ux);
        o.y = xmul(r, uy);
        o.z = xmul(r, uz);
    }
    else if (p.g.kind == 2)
    {
        // VoronoiMeshSnapshot::generatePosition (VoronoiMeshSnapshot.cpp:1007-1020): positions in the
        // cell's enclosing box (Random::position, x, y, z drawn in that order) until one lies at
        // least as close to the cell's site as to every neighbouring site (isPointClosestTo,
        // :879-887, squared distances (r - site).norm2())
        const double* bb = p.g.vBox + 6 * static_cast<size_t>(m);
        const double* sm = p.g.vSites + 3 * static_cast<size_t>(m);
        auto dist2 = [](const double* q, double x, double y, double z) {
            double dx = xsub(x, q[0]), dy = xsub(y, q[1]), dz = xsub(z, q[2]);
            return xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
        };
        for (int tries = 0; tries < 10000; ++tries)
        {
            double fx = rng.uniform(), fy = rng.uniform(), fz = rng.uniform();
            o.x = xadd(bb[0], xmul(fx, xsub(bb[3], bb[0])));
            o.y = xadd(bb[1], xmul(fy, xsub(bb[4], bb[1])));
            o.z = xadd(bb[2], xmul(fz, xsub(bb[5], bb[2])));
            double target = dist2(sm, o.x, o.y, o.z);
            bool closest = true;
            for (int e = p.g.vNbBegin[m]; e < p.g.vNbBegin[m + 1] && closest; ++e)
            {
                int id = p.g.vNb[e];
                if (id >= 0 && dist2(p.g.vSites + 3 * static_cast<size_t>(id), o.x, o.y, o.z) < target) closest = false;
            }
            if (closest) break;
        }
    }
        else if (p.g.kind >= 5 && p.g.kind <= 8)
    {
        // the cylindrical and spherical grids' randomPositionInCell (Cylinder2DSpatialGrid.cpp:95-106,
        // Sphere2DSpatialGrid.cpp:102-113, Sphere3DSpatialGrid.cpp:146-157,
        // Cylinder3DSpatialGrid.cpp:133-144) with getCoords' bin indices and Position's cylindrical
        // and spherical constructors (SKIRT/utils/Position.cpp:21-43)
        const double twoPi = 2.0 * M_PI;
        if (p.g.kind == 5 || p.g.kind == 8)
        {
            int i, j = 0, k;
            const double *Rv, *zv;
            if (p.g.kind == 5)
            {
                i = m / p.g.cNz;
                k = m % p.g.cNz;
                Rv = p.g.cRv;
                zv = p.g.czv;
            }
            else
            {
                i = m / (p.g.c3Np * p.g.c3Nz);
                j = (m / p.g.c3Nz) % p.g.c3Np;
                k = m % p.g.c3Nz;
                Rv = p.g.c3r;
                zv = p.g.c3z;
            }
            double R0 = Rv[i], R1 = Rv[i + 1], z0 = zv[k], z1 = zv[k + 1];
            double R = sqrt(xadd(xmul(R0, R0), xmul(xmul(xsub(R1, R0), xadd(R1, R0)), rng.uniform())));
            double phi = p.g.kind == 5 ? xmul(twoPi, rng.uniform())
                                       : xadd(p.g.c3p[j], xmul(xsub(p.g.c3p[j + 1], p.g.c3p[j]), rng.uniform()));
            double z = xadd(z0, xmul(xsub(z1, z0), rng.uniform()));
            o.x = xmul(R, cos(phi));
            o.y = xmul(R, sin(phi));
            o.z = z;
        }
        else
        {
            int i, j, k = 0;
            const double *rv, *tv;
            if (p.g.kind == 6)
            {
                i = m / p.g.s2Nt;
                j = m % p.g.s2Nt;
                rv = p.g.s2r;
                tv = p.g.s2t;
            }
            else
            {
                i = m / (p.g.s3Nt * p.g.s3Np);
                j = (m / p.g.s3Np) % p.g.s3Nt;
                k = m % p.g.s3Np;
                rv = p.g.s3r;
                tv = p.g.s3t;
            }
            double r0 = rv[i], r1 = rv[i + 1], t0 = tv[j], t1 = tv[j + 1];
            double d3 = xmul(xsub(r1, r0), xadd(xadd(xmul(r1, r1), xmul(r1, r0)), xmul(r0, r0)));
            double r = cbrt(xadd(xmul(xmul(r0, r0), r0), xmul(d3, rng.uniform())));
            double c0 = cos(t0);
            double theta = acos(xadd(c0, xmul(xsub(cos(t1), c0), rng.uniform())));
            double phi = p.g.kind == 6 ? xmul(twoPi, rng.uniform())
                                       : xadd(p.g.s3p[k], xmul(xsub(p.g.s3p[k + 1], p.g.s3p[k]), rng.uniform()));
            double st = sin(theta);
            o.x = xmul(xmul(r, st), cos(phi));
            o.y = xmul(xmul(r, st), sin(phi));
            o.z = xmul(r, cos(theta));
        }
    }
    else
    {
        // the cell box (Random::position, Box::fracPos): Cartesian borders, or the extent of the
        // octree or adaptive-mesh leaf
        double b0, b1, b2, b3, b4, b5;
        if (p.g.kind == 0)
        {
            int i = m / (p.g.nz * p.g.ny), j = (m / p.g.nz) % p.g.ny, k = m % p.g.nz;
            b0 = p.g.xb[i]; b1 = p.g.yb[j]; b2 = p.g.zb[k];
            b3 = p.g.xb[i + 1]; b4 = p.g.yb[j + 1]; b5 = p.g.zb[k + 1];
        }
        else
        {
            const double* bb = p.g.tBounds + 6 * static_cast<size_t>(S.cellNode[m]);
            b0 = bb[0]; b1 = bb[1]; b2 = bb[2]; b3 = bb[3]; b4 = bb[4]; b5 = bb[5];
        }
        double fx = rng.uniform(), fy = rng.uniform(), fz = rng.uniform();
        o.x = xadd(b0, xmul(fx, xsub(b3, b0)));
        o.y = xadd(b1, xmul(fy, xsub(b4, b1)));
        o.z = xadd(b2, xmul(fz, xsub(b5, b2)));
    }
    isotropicDirection(rng, o.kx, o.ky, o.kz);
    o.lambda = lambda;
    o.L = xmul(xmul(S.Lpk, ws), w);
    return o;
}

// SourceSystem::launch -> NormalizedSource::launch -> PointSource / GeometricSource
// (SourceSystem.cpp, NormalizedSource.cpp:73-110, SepAxGeometry.cpp:11-19, SpheGeometry.cpp:25-32,
// ExpDiskGeometry.cpp:46-69, LogWavelengthDistribution.cpp:31-34, Random.cpp:121-207)
SKG_D Launched launchPacket(const Scene& p, unsigned long long hist, Rng& rng)
{
    if (p.sec) return launchSecondary(p, hist, rng);
    int h = 0;
    for (int q = 1; q < p.nsrc; ++q)
        if (p.src[q].first <= hist) h = q;
    const SourceDev& S = p.src[h];
    Launched o;
    double L = S.Lpk;
    double lambda;
    if (S.specModel == 0)
    {
        int j = min(S.tsize - 1, static_cast<int>(rng.uniform() * S.tsize));
        lambda = p.tabL[S.toff + j];
        L *= p.tabA[S.toff + j];
    }
    else
    {
        const double* lv = p.tabL + S.toff;
        const double* pv = p.tabA + S.toff;
        const double* Pv = p.tabB + S.toff;
        int n = S.tsize;
        double xi = S.xi;
        bool fromSed = (xi <= 0.) || (rng.uniform() > xi);
        if (fromSed)
        {
            double X = rng.uniform();
            int i = locateClip(Pv, n, X);
            double alpha = log(pv[i + 1] / pv[i]) / log(lv[i + 1] / lv[i]);
            lambda = lv[i] * gexp(-alpha, (X - Pv[i]) / (pv[i] * lv[i]));
        }
        else
        {
            double lmin = log(S.bmin), lw = log(S.bmax) - log(S.bmin);
            lambda = exp(lmin + lw * rng.uniform());
        }
        if (xi > 0.)
        {
            double s = 0.;
            if (lambda >= lv[0] && lambda <= lv[n - 1])
            {
                int i = min(n - 2, max(0, upperBound(lv, n, lambda) - 1));
                double a = log(pv[i + 1] / pv[i]) / log(lv[i + 1] / lv[i]);
                s = pv[i] * pow(lambda / lv[i], a);
            }
            double b = (lambda >= S.bmin && lambda <= S.bmax) ? 1. / ((log(S.bmax) - log(S.bmin)) * lambda) : 0.;
            L *= (s > 0.) ? s / ((1 - xi) * s + xi * b) : 0.;
        }
    }
    o.lambda = lambda;
    o.L = L;
    if (S.posModel == 0)
    {
        o.x = S.pos[0]; o.y = S.pos[1]; o.z = S.pos[2];
    }
    else if (S.posModel == 1)
    {
        double hR = S.geom[0], hz = S.geom[1], Rmin = S.geom[2], Rmax = S.geom[3], zmax = S.geom[4];
        double R = 0.;
        for (int t = 0; t < 1000; ++t)
        {
            double X = rng.uniform();
            R = hR * (-1.0 - lambertWm1((X - 1.0) / M_E));
            if (!((Rmax > 0.0 && R >= Rmax) || R <= Rmin)) break;
        }
        double phi = 2.0 * M_PI * rng.uniform();
        double z = 0.;
        for (int t = 0; t < 1000; ++t)
        {
            double X = rng.uniform();
            z = (X <= 0.5) ? hz * log(2.0 * X) : -hz * log(2.0 * (1.0 - X));
            if (!(zmax > 0.0 && fabs(z) >= zmax)) break;
        }
        o.x = S.pos[0] + R * cos(phi);
        o.y = S.pos[1] + R * sin(phi);
        o.z = S.pos[2] + z;
    }
    else
    {
        double X = rng.uniform();
        const double* rv = p.radR + S.roff;
        const double* Pv = p.radP + S.roff;
        double r;
        if (S.posModel == 3)
        {
            // SersicFunction::inverseMass: NR::clampedValue<NR::interpolateLogLog>(X, M, s), times the scale
            r = S.geom[0] * clampedLogLog(Pv, rv, S.rsize, X);
        }
        else
        {
            int i = locateClip(Pv, S.rsize, X);
            r = rv[i] + (X - Pv[i]) / (Pv[i + 1] - Pv[i]) * (rv[i + 1] - rv[i]);
        }
        double ux, uy, uz;
        isotropicDirection(rng, ux, uy, uz);
        o.x = S.pos[0] + r * ux;
        o.y = S.pos[1] + r * uy;
        o.z = S.pos[2] + r * uz;
    }
    isotropicDirection(rng, o.kx, o.ky, o.kz);
    return o;
}

// FrameInstrument::pixelOnDetector (FrameInstrument.cpp:117-136)
SKG_D int framePixel(const InstrDev& in, double x, double y, double z)
{
    double xpp = -in.sp * x + in.cp * y;
    double ypp = -in.cp * in.ct * x - in.sp * in.ct * y + in.st * z;
    double xp = in.co * xpp - in.so * ypp;
    double yp = in.so * xpp + in.co * ypp;
    int i = static_cast<int>(floor((xp - in.xpmin) / in.xpsiz));
    int j = static_cast<int>(floor((yp - in.ypmin) / in.ypsiz));
    if (i < 0 || i >= in.npx || j < 0 || j >= in.npy) return -1;
    return i + in.npx * j;
}

// ApertureInstrument::isInsideAperture (ApertureInstrument.cpp:25-44): the position projected with
// inclination and azimuth (no roll) within the aperture radius
SKG_D bool insideAperture(const InstrDev& in, double x, double y, double z)
{
    if (!(in.apR2 > 0.)) return true;
    double xpp = -in.sp * x + in.cp * y;
    double ypp = -in.cp * in.ct * x - in.sp * in.ct * y + in.st * z;
    return !(xpp * xpp + ypp * ypp > in.apR2);
}

// does any instrument of the observer group starting at i0 record a packet at (x,y,z)?
SKG_D bool groupNeedsTau(const Scene& p, int i0, double x, double y, double z)
{
    for (int i = i0; i < p.ninstr && (i == i0 || p.instr[i].same); ++i)
    {
        const InstrDev& in = p.instr[i];
        if (in.kind == 1 && insideAperture(in, x, y, z)) return true;
        if (in.kind == 0 && framePixel(in, x, y, z) >= 0) return true;
    }
    return false;
}

SKG_D int nextGroup(const Scene& p, int i0)
{
    int j = i0 + 1;
    while (j < p.ninstr && p.instr[j].same) ++j;
    return j;
}

// the albedo of the interaction cell (MediumSystem::albedoForScattering, MediumSystem.cpp:793-837)
SKG_D double albedoAt(const Scene& p, int m, double ssca, double sext)
{
    double n = p.dens[m];
    double ksca = n > 0. ? n * ssca : 0.;
    double kext = n > 0. ? n * sext : 0.;
    return kext > 0. ? ksca / kext : 0.;
}

// HG scattering (DustMix::performScattering, DustMix.cpp:490-546)
SKG_D void scatterHG(Rng& rng, double g, double& kx, double& ky, double& kz)
{
    if (fabs(g) < 1e-6)
    {
        isotropicDirection(rng, kx, ky, kz);
    }
    else
    {
        double f = ((1.0 - g) * (1.0 + g)) / (1.0 - g + 2.0 * g * rng.uniform());
        double costheta = (1.0 + g * g - f * f) / (2.0 * g);
        rotateDirection(rng, costheta, kx, ky, kz);
    }
}

}  // namespace skg
