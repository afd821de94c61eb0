// The photon-packet life cycle as one persistent sm_100a kernel.
//
// Each lane owns one history at a time and runs the reference life cycle
// (MonteCarloSimulation::performLifeCycle, SKIRT/core/MonteCarloSimulation.cpp:614-694) as a state
// machine whose states are the traversals of that life cycle:
//   S_PEEL   peel-off towards one observer: optical depth to the domain edge
//            (FluxRecorder::detect -> MediumSystem::getExtinctionOpticalDepth, MediumSystem.cpp:2328-2443)
//   S_PROP1  forced scattering, first pass: cumulative optical depth of the complete path with
//            radiation-field storage (setExtinctionOpticalDepths :1785-1846, storeRadiationField
//            MonteCarloSimulation.cpp:888-957)
//   S_PROP2  forced scattering, second pass: interaction point of the sampled optical depth
//            (simulateForcedPropagation :1492-1546, SpatialGridPath::findInteractionPoint :161-203)
//   S_FREE   non-forced propagation (simulateNonForcedPropagation :1996-2030,
//            MediumSystem::setInteractionPointUsingExtinction :2005-2150)
// Every loop iteration advances each lane's current traversal by exactly one cell crossing, so the
// lanes of a warp execute the (uniform) crossing code together; the short transition code between
// traversals (launch, detection, forced sampling, scattering) runs for the lanes whose traversal
// ended. Lanes that finish a history take a new one at the top of the next iteration; one elected
// lane per warp claims a batch of history indices with a single atomic.
//
// Tallies are FP64: peel-off detections and radiation-field updates are reduced among the lanes of
// a warp that hit the same address (__match_any_sync) before one atomicAdd. Per-history statistics
// (sum w^k) are grouped per lane in a small buffer and flushed at the end of the history.
#pragma once

#include "grids.cuh"

namespace skg {

constexpr int MAX_INSTR = 16;
constexpr int STATS_CAP = 48;
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
    double* ifu;        // total, nbins*npix (frame) ; size 0 for SED
    double* sed;        // total, nbins (SED) ; null for frame
    double* ifuComp;    // 3 planes: transparent, direct, scattered
    double* sedComp;
    double* ifuStats;   // 5 planes
    double* sedStats;
};

struct LCParams
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

    int rfOn;
    int nrf;
    int rfNb;
    const double* rfB;
    const int* rfEll;
    double* rf;

    int forced, minScatt, peel;
    double minWeightRed, pathLengthBias;
    unsigned long long seed;

    unsigned long long first, count, npp;
    unsigned long long* workCounter;
    unsigned long long* counters;  // histories, crossings, scatterings, detections, rfStores, statsOverflows
    int* errFlag;
};

enum LaneStage { S_FETCH = 0, S_DONE = 1, S_PEEL = 2, S_PROP1 = 3, S_PROP2 = 4, S_FREE = 5 };

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

// generalized exponential SpecialFunctions::gexp(p, x) (SKIRT/utils/SpecialFunctions.cpp:822-836),
// the inverse of the generalized logarithm used by Random::cdfLogLog (Random.cpp:200-207)
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

struct Lane
{
    int stage;
    unsigned long long hist;
    Rng rng;
    // packet
    double rx, ry, rz, kx, ky, kz;
    double L, lambda, Lthresh;
    int nscatt;
    int ellMix, ellRF;
    double sext, ssca, gHG;
    // current traversal
    double tau, s, tau0, s0, tauPath, tauInt, lnExtBeg, extBeg;
    int lastM;
    double lastS;
    int nseg;
    int guard;
    // peel-off
    int peelGroup;      // first instrument index of the current observer group
    int peelScatter;    // 0 emission, 1 scattering
    double peelL;
    // statistics buffer (per history)
    int nstat;
    int statOverflow;
};

template<class Walker>
struct LifeCycle
{
    const LCParams& p;
    Lane& ln;
    Walker& w;
    unsigned long long cCross, cScatt, cDetect, cRf, cOverflow;

    SKG_D LifeCycle(const LCParams& pp, Lane& l, Walker& ww)
        : p(pp), ln(l), w(ww), cCross(0), cScatt(0), cDetect(0), cRf(0), cOverflow(0)
    {}

    SKG_D void raiseError(int code) { atomicOr(p.errFlag, code); }

    // ---------------- statistics buffer ----------------
    unsigned long long skey[STATS_CAP];
    double sw[STATS_CAP];

    SKG_D void flushStats()
    {
        for (int a = 0; a < ln.nstat; ++a)
        {
            if (sw[a] != sw[a]) continue;  // NaN marks a consumed entry
            unsigned long long key = skey[a];
            double wsum = sw[a];
            for (int b = a + 1; b < ln.nstat; ++b)
            {
                if (skey[b] == key)
                {
                    wsum += sw[b];
                    sw[b] = __longlong_as_double(0x7ff8000000000000ULL);
                }
            }
            int i = static_cast<int>(key >> 48);
            int ell = static_cast<int>((key >> 24) & 0xFFFFFF);
            int l = static_cast<int>(key & 0xFFFFFF) - 1;
            const InstrDev& in = p.instr[i];
            double wn = 1.;
            if (l < 0)
            {
                for (int k = 0; k <= 4; ++k)
                {
                    atomicAdd(in.sedStats + static_cast<size_t>(k) * in.nbins + ell, wn);
                    wn *= wsum;
                }
            }
            else
            {
                size_t plane = static_cast<size_t>(in.npx) * in.npy * in.nbins;
                size_t lell = static_cast<size_t>(l) + static_cast<size_t>(ell) * in.npx * in.npy;
                for (int k = 0; k <= 4; ++k)
                {
                    atomicAdd(in.ifuStats + k * plane + lell, wn);
                    wn *= wsum;
                }
            }
        }
        ln.nstat = 0;
    }

    SKG_D void addStat(int i, int ell, int l, double v)
    {
        if (ln.nstat == STATS_CAP)
        {
            if (!ln.statOverflow) cOverflow++;
            ln.statOverflow = 1;
            flushStats();
        }
        skey[ln.nstat] = (static_cast<unsigned long long>(i) << 48) | (static_cast<unsigned long long>(ell) << 24)
                         | static_cast<unsigned long long>(l + 1);
        sw[ln.nstat] = v;
        ln.nstat++;
    }

    // ---------------- launch (SourceSystem::launch, NormalizedSource::launch) ----------------
    SKG_D void launch()
    {
        // source for this history: last source whose first index <= hist
        int h = 0;
        for (int q = 1; q < p.nsrc; ++q)
            if (p.src[q].first <= ln.hist) h = q;
        const SourceDev& S = p.src[h];
        ln.rng.start(p.seed, ln.hist);
        ln.nscatt = 0;
        ln.nstat = 0;
        ln.statOverflow = 0;
        double L = S.Lpk;
        double lambda;
        if (S.specModel == 0)
        {
            // oligochromatic: uniform choice among the discrete wavelengths with weight s/b
            int j = min(S.tsize - 1, static_cast<int>(ln.rng.uniform() * S.tsize));
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
            bool fromSed = (xi <= 0.) || (ln.rng.uniform() > xi);
            if (fromSed)
            {
                // Random::cdfLogLog on the SED table
                double X = ln.rng.uniform();
                int i = locateClip(Pv, n, X);
                double alpha = log(pv[i + 1] / pv[i]) / log(lv[i + 1] / lv[i]);
                lambda = lv[i] * gexp(-alpha, (X - Pv[i]) / (pv[i] * lv[i]));
            }
            else
            {
                // LogWavelengthDistribution::generateWavelength (LogWavelengthDistribution.cpp:31-34)
                double lmin = log(S.bmin), lw = log(S.bmax) - log(S.bmin);
                lambda = exp(lmin + lw * ln.rng.uniform());
            }
            if (xi > 0.)
            {
                // specific luminosity: log-log interpolation of the normalised pdf
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
        ln.lambda = lambda;
        ln.L = L;
        // position
        if (S.posModel == 0)
        {
            ln.rx = S.pos[0]; ln.ry = S.pos[1]; ln.rz = S.pos[2];
        }
        else if (S.posModel == 1)
        {
            // SepAxGeometry::generatePosition with ExpDiskGeometry::randomCylRadius / randomZ
            double hR = S.geom[0], hz = S.geom[1], Rmin = S.geom[2], Rmax = S.geom[3], zmax = S.geom[4];
            double R = 0.;
            for (int gtry = 0; gtry < 1000; ++gtry)
            {
                double X = ln.rng.uniform();
                R = hR * (-1.0 - lambertWm1((X - 1.0) / M_E));
                if (!((Rmax > 0.0 && R >= Rmax) || R <= Rmin)) break;
            }
            double phi = 2.0 * M_PI * ln.rng.uniform();
            double z = 0.;
            for (int gtry = 0; gtry < 1000; ++gtry)
            {
                double X = ln.rng.uniform();
                z = (X <= 0.5) ? hz * log(2.0 * X) : -hz * log(2.0 * (1.0 - X));
                if (!(zmax > 0.0 && fabs(z) >= zmax)) break;
            }
            ln.rx = S.pos[0] + R * cos(phi);
            ln.ry = S.pos[1] + R * sin(phi);
            ln.rz = S.pos[2] + z;
        }
        else
        {
            // SpheGeometry::generatePosition: radius from the tabulated cumulative mass, isotropic direction
            double X = ln.rng.uniform();
            const double* rv = p.radR + S.roff;
            const double* Pv = p.radP + S.roff;
            int i = locateClip(Pv, S.rsize, X);
            double r = rv[i] + (X - Pv[i]) / (Pv[i + 1] - Pv[i]) * (rv[i + 1] - rv[i]);
            double ux, uy, uz;
            isotropicDirection(ln.rng, ux, uy, uz);
            ln.rx = S.pos[0] + r * ux;
            ln.ry = S.pos[1] + r * uy;
            ln.rz = S.pos[2] + r * uz;
        }
        isotropicDirection(ln.rng, ln.kx, ln.ky, ln.kz);
        ln.Lthresh = ln.L / p.minWeightRed;
        // wavelength-dependent quantities are constant during a history (no kinematics)
        if (p.nmix > 0)
        {
            ln.ellMix = max(0, locateClip(p.mixLb, p.nmix, lambda));  // a one-entry table has a single bin
            ln.sext = p.mixExt[ln.ellMix];
            ln.ssca = p.mixSca[ln.ellMix];
            ln.gHG = p.mixG[ln.ellMix];
        }
        ln.ellRF = p.rfOn ? wlgBin(p.rfB, p.rfNb, p.rfEll, lambda) : -1;
    }

    // Lambert W, branch -1, for x in [-1/e, 0): Halley iteration from a series/log initial guess
    SKG_D static double lambertWm1(double x)
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

    // ---------------- traversal starts ----------------
    SKG_D void startRay(double ux, double uy, double uz)
    {
        w.start(p.g, ln.rx, ln.ry, ln.rz, ux, uy, uz);
        ln.tau = 0.;
        ln.s = 0.;
        ln.nseg = 0;
        ln.guard = 0;
        ln.lastM = -1;
        ln.lastS = 0.;
    }

    SKG_D void beginProp()
    {
        if (p.forced)
        {
            ln.stage = S_PROP1;
            ln.lnExtBeg = 0.;
            ln.extBeg = 1.;
        }
        else
        {
            ln.stage = S_FREE;
            ln.tauInt = -log(ln.rng.uniform());
        }
        startRay(ln.kx, ln.ky, ln.kz);
    }

    // pixel of a frame instrument (FrameInstrument::pixelOnDetector, FrameInstrument.cpp:117-136)
    SKG_D int framePixel(const InstrDev& in) const
    {
        double x = ln.rx, y = ln.ry, z = ln.rz;
        double xpp = -in.sp * x + in.cp * y;
        double ypp = -in.cp * in.ct * x - in.sp * in.ct * y + in.st * z;
        double xp = in.co * xpp - in.so * ypp;
        double yp = in.so * xpp + in.co * ypp;
        int i = static_cast<int>(floor((xp - in.xpmin) / in.xpsiz));
        int j = static_cast<int>(floor((yp - in.ypmin) / in.ypsiz));
        if (i < 0 || i >= in.npx || j < 0 || j >= in.npy) return -1;
        return i + in.npx * j;
    }

    // does any instrument of the observer group starting at i0 record something for this packet?
    SKG_D bool groupNeedsTau(int i0) const
    {
        for (int i = i0; i < p.ninstr && (i == i0 || p.instr[i].same); ++i)
        {
            const InstrDev& in = p.instr[i];
            if (in.kind == 1) return true;
            if (framePixel(in) >= 0) return true;
        }
        return false;
    }

    // start the peel-off traversal for the next observer group at or after i0; returns false if none left
    SKG_D bool beginPeelGroup(int i0)
    {
        for (int i = i0; i < p.ninstr; ++i)
        {
            if (i != i0 && p.instr[i].same) continue;  // inside a group already handled
            if (!groupNeedsTau(i))
            {
                // skip the group
                int j = i + 1;
                while (j < p.ninstr && p.instr[j].same) ++j;
                i = j - 1;
                continue;
            }
            const InstrDev& in = p.instr[i];
            ln.peelGroup = i;
            if (ln.peelScatter)
            {
                double costheta = ln.kx * in.kobs[0] + ln.ky * in.kobs[1] + ln.kz * in.kobs[2];
                ln.peelL = ln.L * phaseHG(ln.gHG, costheta);
            }
            else
            {
                ln.peelL = ln.L;
            }
            ln.stage = S_PEEL;
            startRay(in.kobs[0], in.kobs[1], in.kobs[2]);
            return true;
        }
        return false;
    }

    // FluxRecorder::detect for every instrument of the current observer group (FluxRecorder.cpp:372-538)
    SKG_D void detectGroup()
    {
        double ext = exp(-ln.tau);
        int numScatt = ln.nscatt + (ln.peelScatter ? 1 : 0);
        int i0 = ln.peelGroup;
        for (int i = i0; i < p.ninstr && (i == i0 || p.instr[i].same); ++i)
        {
            const InstrDev& in = p.instr[i];
            int l = in.kind == 0 ? framePixel(in) : -1;
            if (in.kind == 0 && l < 0) continue;
            int ell = wlgBin(p.wlgB + in.woff, in.wnb, p.wlgEll + in.woff, ln.lambda);
            if (ell < 0) continue;
            double L = ln.peelL;
            double Lext = L * ext;
            cDetect++;
            if (in.kind == 0)
            {
                size_t npix = static_cast<size_t>(in.npx) * in.npy;
                size_t idx = static_cast<size_t>(l) + static_cast<size_t>(ell) * npix;
                atomicAddAgg(in.ifu + idx, Lext);
                if (in.comps)
                {
                    size_t plane = npix * in.nbins;
                    if (numScatt == 0)
                    {
                        atomicAddAgg(in.ifuComp + idx, L);
                        atomicAddAgg(in.ifuComp + plane + idx, Lext);
                    }
                    else
                        atomicAddAgg(in.ifuComp + 2 * plane + idx, Lext);
                }
            }
            else
            {
                atomicAddAgg(in.sed + ell, Lext);
                if (in.comps)
                {
                    if (numScatt == 0)
                    {
                        atomicAddAgg(in.sedComp + ell, L);
                        atomicAddAgg(in.sedComp + in.nbins + ell, Lext);
                    }
                    else
                        atomicAddAgg(in.sedComp + 2 * in.nbins + ell, Lext);
                }
            }
            if (in.stats) addStat(i, ell, l, Lext);
        }
    }

    // HG scattering (DustMix::performScattering, DustMix.cpp:490-546) and PhotonPacket::scatter
    SKG_D void scatter()
    {
        if (ln.nscatt >= MAX_SCATT_EVENTS)
        {
            // a history that never meets its termination criterion (e.g. albedo 1 in a thick medium)
            raiseError(8);
            ln.L = 0.;
        }
        double g = ln.gHG;
        if (fabs(g) < 1e-6)
        {
            isotropicDirection(ln.rng, ln.kx, ln.ky, ln.kz);
        }
        else
        {
            double f = ((1.0 - g) * (1.0 + g)) / (1.0 - g + 2.0 * g * ln.rng.uniform());
            double costheta = (1.0 + g * g - f * f) / (2.0 * g);
            rotateDirection(ln.rng, costheta, ln.kx, ln.ky, ln.kz);
        }
        ln.nscatt++;
        cScatt++;
    }

    SKG_D void endHistory()
    {
        if (ln.nstat) flushStats();
        ln.stage = S_FETCH;
    }

    // after an interaction point has been reached: weight, position, termination, peel-off/scatter
    SKG_D void afterInteraction(int mInt, double sInt, bool forcedPath)
    {
        if (mInt < 0)
        {
            raiseError(2);
            endHistory();
            return;
        }
        double n = p.dens[mInt];
        double ksca = n > 0. ? n * ln.ssca : 0.;
        double kext = n > 0. ? n * ln.sext : 0.;
        double albedo = kext > 0. ? ksca / kext : 0.;
        if (forcedPath)
            ln.L *= -expm1(-ln.tauPath) * albedo;
        else
            ln.L *= albedo;
        ln.rx += sInt * ln.kx;
        ln.ry += sInt * ln.ky;
        ln.rz += sInt * ln.kz;
        if (ln.L <= 0 || (forcedPath && ln.L <= ln.Lthresh && ln.nscatt >= p.minScatt))
        {
            endHistory();
            return;
        }
        if (p.peel && p.ninstr > 0)
        {
            ln.peelScatter = 1;
            if (beginPeelGroup(0)) return;
        }
        scatter();
        beginProp();
    }

    // one loop iteration for this lane: one crossing of the current traversal + transitions
    SKG_D void step()
    {
        bool got = w.next(p.g);
        if (got) cCross++;
        if (++ln.guard > (1 << 22))
        {
            raiseError(4);
            got = false;
        }
        switch (ln.stage)
        {
            case S_PEEL:
            {
                if (got)
                {
                    if (w.m >= 0)
                    {
                        ln.tau = xadd(ln.tau, xmul(xmul(ln.sext, p.dens[w.m]), w.ds));
                        double taumax = log(ln.peelL) + 745.;
                        if (ln.tau >= taumax)
                        {
                            ln.tau = INFINITY;
                            got = false;
                        }
                    }
                    if (got) return;
                }
                // traversal complete: detect in this observer group, then the next group
                detectGroup();
                int j = ln.peelGroup + 1;
                while (j < p.ninstr && p.instr[j].same) ++j;
                if (beginPeelGroup(j)) return;
                if (ln.peelScatter) scatter();
                beginProp();
                return;
            }
            case S_PROP1:
            {
                if (got)
                {
                    if (w.ds > 0.)
                    {
                        int mm = w.m;
                        if (mm >= 0) ln.tau = xadd(ln.tau, xmul(xmul(ln.sext, p.dens[mm]), w.ds));
                        ln.nseg++;
                        if (p.rfOn && ln.ellRF >= 0)
                        {
                            double lnExtEnd = -ln.tau;
                            double extEnd = exp(lnExtEnd);
                            if (mm >= 0)
                            {
                                double extMean = lnmean4(extEnd, ln.extBeg, lnExtEnd, ln.lnExtBeg);
                                double Lds = ln.L * extMean * w.ds;
                                atomicAdd(p.rf + static_cast<size_t>(mm) * p.nrf + ln.ellRF, Lds);
                                cRf++;
                            }
                            ln.lnExtBeg = lnExtEnd;
                            ln.extBeg = extEnd;
                        }
                    }
                    return;
                }
                // complete path known: sample the interaction optical depth (simulateForcedPropagation)
                double taupath = ln.nseg ? ln.tau : 0.;
                if (taupath <= 0.)
                {
                    ln.L *= 0.;
                    endHistory();
                    return;
                }
                ln.tauPath = taupath;
                double xi = p.pathLengthBias;
                double t;
                if (xi == 0.)
                {
                    t = exponCutoff(ln.rng, taupath);
                }
                else
                {
                    t = ln.rng.uniform() < xi ? ln.rng.uniform() * taupath : exponCutoff(ln.rng, taupath);
                    double pp = -exp(-t) / expm1(-taupath);
                    double q = (1.0 - xi) * pp + xi / taupath;
                    ln.L *= pp / q;
                }
                ln.tauInt = t;
                ln.stage = S_PROP2;
                startRay(ln.kx, ln.ky, ln.kz);
                return;
            }
            case S_PROP2:
            {
                if (got)
                {
                    if (w.ds > 0.)
                    {
                        double tau0 = ln.tau, s0 = ln.s;
                        if (w.m >= 0) ln.tau = xadd(ln.tau, xmul(xmul(ln.sext, p.dens[w.m]), w.ds));
                        ln.s = xadd(ln.s, w.ds);
                        ln.lastM = w.m;
                        ln.lastS = ln.s;
                        if (ln.tauInt < ln.tau)
                        {
                            // NR::interpolateLinLin (SKIRT/utils/NR.hpp:328-331)
                            double sInt = s0 + ((ln.tauInt - tau0) / (ln.tau - tau0)) * (ln.s - s0);
                            afterInteraction(w.m, sInt, true);
                        }
                    }
                    return;
                }
                // at or beyond the exit optical depth of the last segment: use the last segment
                afterInteraction(ln.lastM, ln.lastS, true);
                return;
            }
            case S_FREE:
            {
                if (got)
                {
                    double tau0 = ln.tau, s0 = ln.s;
                    if (w.m >= 0) ln.tau = xadd(ln.tau, xmul(xmul(ln.sext, p.dens[w.m]), w.ds));
                    ln.s = xadd(ln.s, w.ds);
                    if (ln.tauInt < ln.tau)
                    {
                        double sInt = s0 + ((ln.tauInt - tau0) / (ln.tau - tau0)) * (ln.s - s0);
                        afterInteraction(w.m, sInt, false);
                    }
                    return;
                }
                // the interaction point is outside of the path: the packet escapes
                endHistory();
                return;
            }
            default: return;
        }
    }

    // a freshly fetched history: launch, emission peel-off or first propagation
    SKG_D void begin()
    {
        launch();
        if (!(ln.L > 0))
        {
            endHistory();
            return;
        }
        if (p.peel && p.ninstr > 0)
        {
            ln.peelScatter = 0;
            if (beginPeelGroup(0)) return;
        }
        beginProp();
    }
};

template<class Walker>
__global__ void __launch_bounds__(256) lifecycleKernel(LCParams p)
{
    Lane ln;
    ln.stage = S_FETCH;
    Walker w;
    LifeCycle<Walker> lc(p, ln, w);
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    unsigned long long hists = 0;
    const unsigned long long end = p.first + p.count;

    while (true)
    {
        // warp-aggregated work fetch
        unsigned need = __ballot_sync(FULL, ln.stage == S_FETCH);
        if (need)
        {
            int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(p.workCounter, static_cast<unsigned long long>(__popc(need)));
            base = __shfl_sync(FULL, base, leader);
            if (ln.stage == S_FETCH)
            {
                unsigned long long h = p.first + base + __popc(need & ((1u << lane) - 1));
                if (h < end)
                {
                    ln.hist = h;
                    hists++;
                    lc.begin();
                }
                else
                {
                    ln.stage = S_DONE;
                }
            }
        }
        if (__all_sync(FULL, ln.stage == S_DONE)) break;
        if (ln.stage >= S_PEEL) lc.step();
    }

    // counters: warp reduction then one atomic per warp
    unsigned long long v[6] = {hists, lc.cCross, lc.cScatt, lc.cDetect, lc.cRf, lc.cOverflow};
#pragma unroll
    for (int c = 0; c < 6; ++c)
    {
        unsigned long long x = v[c];
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(FULL, x, off);
        if (lane == 0 && x) atomicAdd(p.counters + c, x);
    }
}

}  // namespace skg
